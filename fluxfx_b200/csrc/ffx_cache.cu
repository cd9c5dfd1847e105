// Bake readback: the preview channels of a step packed into one FP32 staging
// buffer (channel after channel, x-fast), which is exactly the byte layout of
// a playback-cache frame (fluxfx/physics/cache.py:88-101). One launch snapshots
// the solver's fields (FP32, BF16 or the uint8 collider mask) so that a single
// device-to-host copy of the staging buffer, overlapped with the next steps,
// carries the whole frame; the solver's ping-pong buffers are free again as
// soon as this kernel has run.
#include "ffx_host.cuh"

namespace ffx {
namespace {

constexpr int kPackThreads = 256;
constexpr int kMaxPackChannels = 8;

struct PackArgs {
    const void* field[kMaxPackChannels];
    int kind[kMaxPackChannels];   // FFX_F32, FFX_BF16 or FFX_PACK_U8
};

__global__ void __launch_bounds__(kPackThreads) pack_channels_kernel(int64_t count, int channels, PackArgs A,
                                                                     float* __restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int c = 0; c < channels; ++c) {
        float* dst = out + (int64_t)c * count;
        const int kind = A.kind[c];
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
            float v;
            if (kind == FFX_F32) v = __ldg(static_cast<const float*>(A.field[c]) + i);
            else if (kind == FFX_BF16) v = __bfloat162float(static_cast<const __nv_bfloat16*>(A.field[c])[i]);
            else v = (float)__ldg(static_cast<const uint8_t*>(A.field[c]) + i);
            dst[i] = v;
        }
    }
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" int ffx_pack_channels(int64_t count, int channels, const void* const* fields, const int* kinds, float* out,
                                 void* stream) {
    FFX_REQUIRE(count >= 1 && channels >= 1 && channels <= kMaxPackChannels && fields && kinds && out,
                "ffx_pack_channels: invalid arguments (1..%d channels)", kMaxPackChannels);
    PackArgs A = {};
    for (int c = 0; c < channels; ++c) {
        FFX_REQUIRE(fields[c] && (kinds[c] == FFX_F32 || kinds[c] == FFX_BF16 || kinds[c] == FFX_PACK_U8),
                    "ffx_pack_channels: channel %d invalid", c);
        A.field[c] = fields[c];
        A.kind[c] = kinds[c];
    }
    const int64_t want = (count + kPackThreads - 1) / kPackThreads;
    const unsigned blocks = (unsigned)(want < 148 * 8 ? want : 148 * 8);
    pack_channels_kernel<<<blocks, kPackThreads, 0, as_stream(stream)>>>(count, channels, A, out);
    return launch_status("pack_channels_kernel");
}
