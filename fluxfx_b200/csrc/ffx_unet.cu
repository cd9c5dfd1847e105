// Learned pressure warm start: BF16 implicit-GEMM 3D convolutions (forward,
// data gradient, weight gradient), ReLU backward, Adam, and the loss.
//
// Activations are NDHWC bfloat16 (a voxel's channels are contiguous); a tensor
// is addressed through a view (pointer, elements per voxel, first channel), so
// the decoder's concatenation of the upsampled path and the skip connection is
// one buffer that both producers write into and every consumer reads a channel
// range of, without copies.
//
// Forward convolution as a GEMM: rows = output voxels, columns = output
// channels, reduction k = (tap, input channel), A gathered from the input with
// zero padding (implicit im2col), B = weights [k][cout]. Tiles of 128 x 64 x 16
// per block of four warps, a three-stage cp.async pipeline (zero-fill for
// padding and ragged edges), and BF16 tensor-core MMAs (m16n8k16, FP32
// accumulation, fragments via ldmatrix). The transposed 2^3 stride-2
// convolution (decoder up-sampling, and the data gradient of the stride-2
// down-sampling) maps each output voxel 2q + j to tap j of input voxel q: one
// GEMM per parity class j (blockIdx.z). Weight gradients reduce over voxels:
// dW[k][n] = sum_m A[m][k] G[m][n], split over voxel chunks with FP32 atomics.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "ffx_host.cuh"

namespace ffx {
namespace {

using bf16 = __nv_bfloat16;

constexpr int kBM = 128, kBN = 64, kStages = 3, kGemmThreads = 128;
constexpr int kAStride = 24;    // bf16 per A row in shared memory (16 + 8 pad: 48 B, conflict-free ldmatrix)
constexpr int kBStride = 72;    // bf16 per B row (64 + 8 pad: 144 B)
constexpr int kWStride = 136;   // bf16 per A row of the weight-gradient tile (128 + 8 pad: 272 B)

struct View {
    const bf16* p;
    int pitch, offset;
};

struct Conv {
    int batch, id, ih, iw, od, oh, ow;
    int c1, c2, cin, cout, ks, stride, pad, transposed;
    int taps, units_per_tap, k_units;   // reduction in units of 8 channels
    long long rows;                      // GEMM rows: output voxels, or input voxels per parity class
    View in1, in2;
    const bf16* w;
    const float* bias;
    int relu, accumulate;
    bf16* out;
    int out_pitch, out_offset;
    float* out_f32;
    int out_f32_pitch;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int size = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(size));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void ldmatrix_x4(unsigned r[4], const void* smem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(s));
}
__device__ __forceinline__ void ldmatrix_x4_trans(unsigned r[4], const void* smem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(s));
}
__device__ __forceinline__ void mma_bf16(float c[4], const unsigned a[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Position of GEMM row m: the output voxel (convolution) or the input voxel q
// of a parity class (transposed).
struct RowPos {
    int b, z, y, x;
};
__device__ __forceinline__ RowPos decode(long long m, int d, int h, int w) {
    RowPos r;
    r.x = (int)(m % w);
    long long t = m / w;
    r.y = (int)(t % h);
    t /= h;
    r.z = (int)(t % d);
    r.b = (int)(t / d);
    return r;
}

// Address of unit u (8 channels) of GEMM row `pos` in the gathered input, or
// nullptr where the tap falls outside the input (zero padding).
__device__ __forceinline__ const bf16* gather(const Conv& a, const RowPos& pos, int u) {
    const int tap = u / a.units_per_tap;
    const int c = (u - tap * a.units_per_tap) * 8;
    long long vox;
    if (a.transposed) {
        vox = (((long long)pos.b * a.id + pos.z) * a.ih + pos.y) * a.iw + pos.x;
    } else {
        const int ks = a.ks;
        const int dz = tap / (ks * ks), dy = (tap / ks) % ks, dx = tap % ks;
        const int zz = pos.z * a.stride - a.pad + dz, yy = pos.y * a.stride - a.pad + dy,
                  xx = pos.x * a.stride - a.pad + dx;
        if ((unsigned)zz >= (unsigned)a.id || (unsigned)yy >= (unsigned)a.ih || (unsigned)xx >= (unsigned)a.iw)
            return nullptr;
        vox = (((long long)pos.b * a.id + zz) * a.ih + yy) * a.iw + xx;
    }
    if (c < a.c1) return a.in1.p + vox * a.in1.pitch + a.in1.offset + c;
    return a.in2.p + vox * a.in2.pitch + a.in2.offset + (c - a.c1);
}

// Output voxel index of GEMM row m (class j for the transposed form).
__device__ __forceinline__ long long out_voxel(const Conv& a, long long m, int cls) {
    if (!a.transposed) return m;
    const RowPos q = decode(m, a.id, a.ih, a.iw);
    const int z = 2 * q.z + (cls >> 2), y = 2 * q.y + ((cls >> 1) & 1), x = 2 * q.x + (cls & 1);
    return (((long long)q.b * a.od + z) * a.oh + y) * a.ow + x;
}

// ------------------------------------------------------------ forward GEMM
// BN output channels per block (16, 32 or 64, chosen from cout so that narrow
// layers do not multiply padded channels).
template <int BN>
__global__ void __launch_bounds__(kGemmThreads) conv_fwd_kernel(const __grid_constant__ Conv a) {
    constexpr int BS = BN + 8;   // bf16 per B row in shared memory (8 pad: conflict-free ldmatrix)
    __shared__ __align__(128) bf16 sA[kStages][kBM * kAStride];
    __shared__ __align__(128) bf16 sB[kStages][16 * BS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long m0 = (long long)blockIdx.x * kBM;
    const int n0 = blockIdx.y * BN;
    const int cls = blockIdx.z;
    const bf16* W = a.w + (a.transposed ? (size_t)cls * a.cin * a.cout : 0);
    const long long my_row = m0 + tid;
    const bool row_ok = my_row < a.rows;
    const RowPos pos = row_ok ? (a.transposed ? decode(my_row, a.id, a.ih, a.iw) : decode(my_row, a.od, a.oh, a.ow))
                              : RowPos{0, 0, 0, 0};
    const int k_elems = a.k_units * 8;
    const int nk = (a.k_units + 1) / 2;

    auto load = [&](int stage, int kstep) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int u = kstep * 2 + h;
            const bf16* src = (row_ok && u < a.k_units) ? gather(a, pos, u) : nullptr;
            cp_async16(&sA[stage][tid * kAStride + h * 8], src ? src : a.in1.p, src != nullptr);
        }
        if (tid < 2 * BN) {   // 16 rows x BN / 8 units of 8 channels
            const int kr = tid / (BN / 8), nu = (tid % (BN / 8)) * 8;
            const int k = kstep * 16 + kr, n = n0 + nu;
            const bool ok = k < k_elems && n < a.cout;
            cp_async16(&sB[stage][kr * BS + nu], ok ? W + (size_t)k * a.cout + n : W, ok);
        }
    };

    float acc[2][BN / 8][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < BN / 8; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nk) load(s, s);
        cp_async_commit();
    }
    for (int ks = 0; ks < nk; ++ks) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        const int pf = ks + kStages - 1;
        if (pf < nk) load(pf % kStages, pf);
        cp_async_commit();
        const int st = ks % kStages;
        unsigned af[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
            ldmatrix_x4(af[mt], &sA[st][(warp * 32 + mt * 16 + (lane & 15)) * kAStride + (lane >> 4) * 8]);
#pragma unroll
        for (int np = 0; np < BN / 16; ++np) {
            unsigned bf[4];
            ldmatrix_x4_trans(bf, &sB[st][((lane & 7) + ((lane >> 3) & 1) * 8) * BS + np * 16 + (lane >> 4) * 8]);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                mma_bf16(acc[mt][2 * np], af[mt], bf[0], bf[1]);
                mma_bf16(acc[mt][2 * np + 1], af[mt], bf[2], bf[3]);
            }
        }
    }
    cp_async_wait<0>();

    // epilogue: bias, ReLU, optional accumulation, BF16 and/or FP32 stores
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const long long m = m0 + warp * 32 + mt * 16 + (lane >> 2) + half * 8;
            if (m >= a.rows) continue;
            const long long vox = out_voxel(a, m, cls);
#pragma unroll
            for (int nt = 0; nt < BN / 8; ++nt) {
                const int n = n0 + nt * 8 + (lane & 3) * 2;
                if (n >= a.cout) continue;
                float v0 = acc[mt][nt][half * 2], v1 = acc[mt][nt][half * 2 + 1];
                if (a.bias) {
                    v0 += a.bias[n];
                    v1 += a.bias[n + 1];
                }
                if (a.relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                if (a.out) {
                    __nv_bfloat162* o =
                        reinterpret_cast<__nv_bfloat162*>(a.out + vox * a.out_pitch + a.out_offset + n);
                    if (a.accumulate) {
                        const float2 prev = __bfloat1622float2(*o);
                        v0 += prev.x;
                        v1 += prev.y;
                    }
                    *o = __floats2bfloat162_rn(v0, v1);
                }
                if (a.out_f32) {
                    float* o = a.out_f32 + vox * a.out_f32_pitch + n;
                    o[0] = v0;
                    o[1] = v1;
                }
            }
        }
}

// ------------------------------------------------- forward GEMM, tcgen05
// The same implicit GEMM on the 5th-generation tensor cores: one elected
// thread issues tcgen05.mma (kind::f16, M = 128, N = BN, K = 16, BF16 in, FP32
// accumulated in tensor memory) from shared-memory operand descriptors, the
// accumulator tile lives in TMEM for the whole reduction, and the epilogue
// reads it back with tcgen05.ld (one row per thread). Operands are staged by
// cp.async in the canonical no-swizzle core-matrix layouts: A (voxels x k)
// K-major, 8 rows x 16 B per core matrix; B (k x channels) MN-major straight
// from the [k][cout] weights, 8 k-rows x 8 channels per core matrix. A stage
// holds K = 32 (two MMAs); a single mbarrier tracks MMA completion through
// tcgen05.commit. Every wait is bounded: on timeout the kernel records it in
// g_conv_timeouts, stops issuing, and still frees its TMEM.
__device__ int g_conv_timeouts;

constexpr int kTcStages = 3;                     // ring of operand stages (36 KB at BN = 64: six blocks per SM)
constexpr int kTcStageK = 32;                    // two MMA k-steps of 16
constexpr int kTcSpin = 1 << 22;                 // bounded mbarrier polling

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (no swizzle): start, leading- and stride-
// dimension byte offsets (16-byte units), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                      // version
    return d;                                    // base offset 0, layout type 0 (no swizzle)
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (int i = 0; i < kTcSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

template <int BN>
constexpr int tc_smem_bytes() { return kTcStages * (2 * kBM * 16 * 2 + 2 * 16 * BN * 2); }

template <int BN>
__global__ void __launch_bounds__(kGemmThreads) conv_fwd_tc_kernel(const __grid_constant__ Conv a) {
    static_assert(BN == 16 || BN == 32 || BN == 64, "BN");
    constexpr int kAStep = kBM * 16 * 2;             // bytes of A per MMA k-step (128 rows x 16 k)
    constexpr int kBStep = 16 * BN * 2;              // bytes of B per MMA k-step (16 k x BN)
    constexpr int kTmemCols = BN < 32 ? 32 : BN;
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char (*sA)[2 * kAStep] = reinterpret_cast<unsigned char (*)[2 * kAStep]>(tc_smem);
    unsigned char (*sB)[2 * kBStep] =
        reinterpret_cast<unsigned char (*)[2 * kBStep]>(tc_smem + kTcStages * 2 * kAStep);
    __shared__ __align__(8) uint64_t mbar[kTcStages];   // one per stage: its MMAs completed
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long m0 = (long long)blockIdx.x * kBM;
    const int n0 = blockIdx.y * BN;
    const int cls = blockIdx.z;
    const bf16* W = a.w + (a.transposed ? (size_t)cls * a.cin * a.cout : 0);
    const long long my_row = m0 + tid;
    const bool row_ok = my_row < a.rows;
    const RowPos pos = row_ok ? (a.transposed ? decode(my_row, a.id, a.ih, a.iw) : decode(my_row, a.od, a.oh, a.ow))
                              : RowPos{0, 0, 0, 0};
    const int k_elems = a.k_units * 8;
    const int nk = (a.k_units + 3) / 4;              // stages of 4 units (K = 32)

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        abort_flag = 0;
        for (int st = 0; st < kTcStages; ++st)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[st])));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    // A: row `tid`, units u (8 channels) of the stage -> core (row/8, chunk)
    // B: k-row r (0..31) x channel chunk h (BN/8) -> MN-major core matrices
    auto load = [&](int stage, int kstep) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int u = kstep * 4 + c;
            const bf16* src = (row_ok && u < a.k_units) ? gather(a, pos, u) : nullptr;
            unsigned char* dst = sA[stage] + (c >> 1) * kAStep + (tid >> 3) * 256 + (c & 1) * 128 + (tid & 7) * 16;
            cp_async16(dst, src ? src : a.in1.p, src != nullptr);
        }
        constexpr int kBLoads = kTcStageK * (BN / 8);       // 16-byte chunks of B per stage
        for (int q = tid; q < kBLoads; q += kGemmThreads) {
            const int r = q / (BN / 8), h = q % (BN / 8);
            const int k = kstep * kTcStageK + r, n = n0 + h * 8;
            const bool ok = k < k_elems && n < a.cout;
            unsigned char* dst = sB[stage] + (r >> 4) * kBStep + h * 256 + ((r & 15) >> 3) * 128 + (r & 7) * 16;
            cp_async16(dst, ok ? W + (size_t)k * a.cout + n : W, ok);
        }
    };
    // kind::f16, D = F32, A = B = BF16, A K-major, B MN-major, N = BN, M = 128
    const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(kBM >> 4) << 24);

    constexpr int kAhead = 1;                         // stages loaded ahead of the MMAs
#pragma unroll
    for (int st = 0; st < kAhead; ++st) {
        if (st < nk) load(st, st);
        cp_async_commit();
    }
    bool ok = true;
    for (int ks = 0; ks < nk && ok; ++ks) {
        // the prefetch overwrites the stage whose MMAs were issued two iterations ago:
        // wait for that stage's use (kTcStages - kAhead MMA groups may stay in flight)
        const int pf = ks + kAhead;
        const int ps = pf % kTcStages;
        if (pf < nk && pf >= kTcStages) {
            if (!mbar_wait(smem_u32(&mbar[ps]), (uint32_t)(((pf - kTcStages) / kTcStages) & 1))) ok = false;
        }
        if (__syncthreads_or(!ok)) { ok = false; break; }
        if (pf < nk) load(ps, pf);
        cp_async_commit();
        cp_async_wait<kAhead>();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const int st = ks % kTcStages;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const uint64_t da = umma_desc(smem_u32(sA[st] + j * kAStep), 128, 256);
                const uint64_t db = umma_desc(smem_u32(sB[st] + j * kBStep), 128, 256);
                const uint32_t acc = (ks > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(smem_u32(&mbar[st])));
        }
    }
    cp_async_wait<0>();
    // the last commit covers every MMA issued (its stage's barrier, last use)
    const uint32_t last_bar = nk > 0 ? smem_u32(&mbar[(nk - 1) % kTcStages]) : 0u;
    const uint32_t last_parity = nk > 0 ? (uint32_t)(((nk - 1) / kTcStages) & 1) : 0u;
    if (ok && nk > 0 && !mbar_wait(last_bar, last_parity)) ok = false;
    if (!ok && tid == 0) atomicAdd(&g_conv_timeouts, 1);
    if (__syncthreads_or(!ok)) {
        // give MMAs possibly still in flight a bounded grace period before freeing TMEM
        if (nk > 0) mbar_wait(last_bar, last_parity);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;");
        // epilogue: warp w holds TMEM lanes 32w..32w+31 = rows of the tile
        const long long m = m0 + warp * 32 + lane;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(taddr + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < a.rows) {
                const long long vox = out_voxel(a, m, cls);
#pragma unroll
                for (int e = 0; e < 16; e += 2) {
                    const int n = n0 + c0 + e;
                    if (n >= a.cout) continue;
                    float v0 = __uint_as_float(r[e]), v1 = __uint_as_float(r[e + 1]);
                    if (a.bias) {
                        v0 += a.bias[n];
                        v1 += a.bias[n + 1];
                    }
                    if (a.relu) {
                        v0 = fmaxf(v0, 0.f);
                        v1 = fmaxf(v1, 0.f);
                    }
                    if (a.out) {
                        __nv_bfloat162* o =
                            reinterpret_cast<__nv_bfloat162*>(a.out + vox * a.out_pitch + a.out_offset + n);
                        if (a.accumulate) {
                            const float2 prev = __bfloat1622float2(*o);
                            v0 += prev.x;
                            v1 += prev.y;
                        }
                        *o = __floats2bfloat162_rn(v0, v1);
                    }
                    if (a.out_f32) {
                        float* o = a.out_f32 + vox * a.out_f32_pitch + n;
                        o[0] = v0;
                        o[1] = v1;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

// ------------------------------- 3^3 convolution: TMA halo tile + tcgen05
// Stride-1, pad-1 3x3x3 layers without a gather. A work tile is an output
// block of 8 (x) x 16 (y) x bz (z) voxels and BN output channels; its input
// footprint, a 10 x 18 x (bz + 2) halo tile, comes in by one TMA tensor load
// per 8-channel plane (zero-filled outside the grid, which is the padding).
// In shared memory a plane is laid out [z][y][x][8 channels], 16 bytes per
// voxel, so for every tap (dz, dy, dx) the 128 rows (8 x-voxels x 16 y-rows)
// of the A operand are the canonical no-swizzle K-major core matrices of a
// shifted window: start = the tap's first voxel, 8-row groups one halo row
// (160 B) apart, the two 8-channel halves of K = 16 one plane apart. No data
// moves per tap: a K = 16 channel group costs 27 x bz MMAs (M = 128, N = BN)
// on one staged tile. The weights of a group, pre-packed into the MN-major
// core-matrix image of all 27 taps, arrive by one bulk copy with the planes.
//
// The kernel is persistent and warp-specialised: warp 4 (one thread) issues
// the loads of tile after tile into a ring of stages, warp 5 (one thread)
// issues the MMAs into one of two accumulator sets in tensor memory (bz x BN
// FP32 columns each), and warps 0-3 drain the other set (tcgen05.ld, bias,
// ReLU, accumulation, BF16 or FP32 stores), so a tile's loads, its MMAs and
// the previous tile's epilogue overlap. mbarriers hand over stages (full: the
// loads landed; empty: the stage's MMAs completed, by tcgen05.commit) and
// accumulator sets (acc_full by tcgen05.commit, acc_empty by the four
// epilogue warps). Every wait is bounded and also ends when another role has
// given up (a shared abort flag); the block then counts a timeout in
// g_conv_timeouts, lets its copies and MMAs drain (bounded), frees its tensor
// memory and returns.
constexpr int kTmX = 8, kTmY = 16;                   // output tile in x, y (M = 128)
constexpr int kTmHX = kTmX + 2, kTmHY = kTmY + 2;    // halo tile
constexpr int kTmThreads = 192;                      // warps 0-3 epilogue, 4 loads, 5 MMAs
constexpr int kTmMaxStages = 4;
constexpr int kTmSmemLimit = 200 * 1024;             // dynamic shared memory attribute of the kernels

struct TmaConv {
    CUtensorMap act;          // input: (channel, x, y, z, batch), box (8, 10, 18, bz + 2, 1)
    const bf16* wpack;        // packed weights: [cout / BN][groups][27][BN / 8][16][8]
    int batch, d, h, w;       // grid (input = output)
    int cin, cout, groups;    // groups = ceil(cin / 16) channel groups of K = 16
    int bz, tiles_x, tiles_y, tiles_z, nblocks;
    int tiles;                // work tiles: tiles_x * tiles_y * tiles_z * batch * nblocks
    int stages, planes;       // planes loaded per group (1 when cin == 8)
    uint32_t plane;           // bytes of one plane in shared memory (multiple of 128)
    uint32_t stage;           // bytes of one stage: 2 planes + 27 weight tiles
    uint32_t tx;              // bytes a stage's loads deliver
    uint32_t cols;            // tensor-memory columns allocated (2 accumulator sets)
    const float* bias;
    int relu, accumulate;
    bf16* out;
    int out_pitch, out_offset;
    float* out_f32;
    int out_f32_pitch;
};

struct TmTile {
    int nb, x0, y0, z0, b;
};
__device__ __forceinline__ TmTile tm_tile(const TmaConv& P, int t) {
    TmTile r;
    r.nb = t % P.nblocks;
    t /= P.nblocks;
    r.x0 = (t % P.tiles_x) * kTmX;
    t /= P.tiles_x;
    r.y0 = (t % P.tiles_y) * kTmY;
    t /= P.tiles_y;
    r.z0 = (t % P.tiles_z) * P.bz;
    r.b = t / P.tiles_z;
    return r;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Bounded wait that also gives up once another role has set `abort`.
__device__ __forceinline__ bool tm_wait(uint32_t bar, uint32_t parity, const volatile int* abort) {
    for (int i = 0; i < kTcSpin; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 255) == 255 && *abort) return false;
    }
    return false;
}

// The halo planes of group g (channels 16g .. 16g + 15) and its packed weights.
template <int BN>
__device__ __forceinline__ void tm_issue_loads(const TmaConv& P, uint32_t st, uint32_t bar, int g, const TmTile& T) {
    mbar_expect_tx(bar, P.tx);
    const uint64_t map = reinterpret_cast<uint64_t>(&P.act);
    for (int h = 0; h < P.planes; ++h)
        asm volatile(
            "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
            ::"r"(st + h * P.plane), "l"(map), "r"(16 * g + 8 * h), "r"(T.x0 - 1), "r"(T.y0 - 1), "r"(T.z0 - 1),
              "r"(T.b), "r"(bar)
            : "memory");
    constexpr uint32_t kWBytes = 27u * 32u * BN;
    const bf16* src = P.wpack + ((size_t)T.nb * P.groups + g) * (kWBytes / 2);
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(st + 2 * P.plane), "l"(src), "r"(kWBytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tm_mma(uint32_t tmem, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tm_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

// Epilogue of one tile: warp w reads tensor-memory lanes 32w .. 32w + 31 (the
// tile's rows m = 8 y + x) of accumulator set `acc`.
template <int BN>
__device__ __forceinline__ void tm_epilogue(const TmaConv& P, const TmTile& T, uint32_t acc, int warp, int lane) {
    const int m = warp * 32 + lane;
    const int x = T.x0 + (m & 7), y = T.y0 + (m >> 3);
    const uint32_t lane_addr = acc + ((uint32_t)(warp * 32) << 16);
    for (int j = 0; j < P.bz; ++j) {
        const int z = T.z0 + j;
        const bool in = x < P.w && y < P.h && z < P.d;
        const long long vox = (((long long)T.b * P.d + z) * P.h + y) * P.w + x;
#pragma unroll
        for (int c0 = 0; c0 < BN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(lane_addr + (uint32_t)(j * BN + c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (!in) continue;
            const int n = T.nb * BN + c0;
            float v[16];
#pragma unroll
            for (int e = 0; e < 16; ++e) {
                v[e] = __uint_as_float(r[e]);
                if (P.bias) v[e] += __ldg(P.bias + n + e);
                if (P.relu) v[e] = fmaxf(v[e], 0.f);
            }
            if (P.out) {
                uint4* o = reinterpret_cast<uint4*>(P.out + vox * P.out_pitch + P.out_offset + n);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    if (P.accumulate) {
                        const uint4 prev = o[q];
                        const __nv_bfloat162* pv = reinterpret_cast<const __nv_bfloat162*>(&prev);
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float2 f = __bfloat1622float2(pv[e]);
                            v[8 * q + 2 * e] += f.x;
                            v[8 * q + 2 * e + 1] += f.y;
                        }
                    }
                    uint4 pk;
                    __nv_bfloat162* pp = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
                    for (int e = 0; e < 4; ++e) pp[e] = __floats2bfloat162_rn(v[8 * q + 2 * e], v[8 * q + 2 * e + 1]);
                    o[q] = pk;
                }
            }
            if (P.out_f32) {
                float* o = P.out_f32 + vox * P.out_f32_pitch + n;
#pragma unroll
                for (int e = 0; e < 16; ++e) o[e] = v[e];
            }
        }
    }
}

template <int BN>
__global__ void __launch_bounds__(kTmThreads, 1) conv3_tma_kernel(const __grid_constant__ TmaConv P) {
    static_assert(BN == 16 || BN == 32 || BN == 64, "BN");
    extern __shared__ __align__(128) unsigned char tm_smem[];
    __shared__ __align__(8) uint64_t full[kTmMaxStages], empty[kTmMaxStages], acc_full[2], acc_empty[2], drained;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_word;
    volatile int* abort_flag = &abort_word;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t base = (smem_u32(tm_smem) + 127u) & ~127u;
    const uint32_t acc_cols = (uint32_t)(P.bz * BN);
    const int S = P.stages;

    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base)), "r"(P.cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (P.planes == 1) {
        // cin == 8: the second channel half of K is zero in every stage
        for (int s = 0; s < S; ++s)
            for (uint32_t i = tid * 16; i < P.plane; i += kTmThreads * 16)
                asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(base + s * P.stage + P.plane + i),
                             "r"(0u)
                             : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (tid == 0) {
        abort_word = 0;
        for (int s = 0; s < S; ++s) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full[s])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty[s])));
        }
        for (int a = 0; a < 2; ++a) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&acc_full[a])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 4;" ::"r"(smem_u32(&acc_empty[a])));
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&drained)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;

    if (warp == 4) {
        if (lane == 0) {
            // loads: tile after tile, group after group, into the stage ring
            int q = 0;
            for (int t = blockIdx.x; t < P.tiles && !*abort_flag; t += gridDim.x) {
                const TmTile T = tm_tile(P, t);
                for (int g = 0; g < P.groups; ++g, ++q) {
                    const int s = q % S;
                    if (q >= S && !tm_wait(smem_u32(&empty[s]), (uint32_t)(((q / S) - 1) & 1), abort_flag)) {
                        *abort_flag = 1;
                        break;
                    }
                    tm_issue_loads<BN>(P, base + s * P.stage, smem_u32(&full[s]), g, T);
                }
            }
            // the last load of every stage has landed before the block may exit
            for (int k = q > S ? q - S : 0; k < q; ++k) mbar_wait(smem_u32(&full[k % S]), (uint32_t)((k / S) & 1));
        }
    } else if (warp == 5) {
        if (lane == 0) {
            // MMAs: D[set][j] += A(tap, z slice j) x B(tap), 27 taps x bz slices per group
            const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((uint32_t)(BN >> 3) << 17) |
                                   ((uint32_t)(128 >> 4) << 24);
            int q = 0, it = 0;
            for (int t = blockIdx.x; t < P.tiles && !*abort_flag; t += gridDim.x, ++it) {
                const int a = it & 1;
                if (it >= 2 && !tm_wait(smem_u32(&acc_empty[a]), (uint32_t)(((it >> 1) - 1) & 1), abort_flag)) {
                    *abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t d0 = tmem + (uint32_t)a * acc_cols;
                bool ok = true;
                for (int g = 0; g < P.groups; ++g, ++q) {
                    const int s = q % S;
                    if (!tm_wait(smem_u32(&full[s]), (uint32_t)((q / S) & 1), abort_flag)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    const uint32_t st = base + s * P.stage;
                    const uint64_t da0 = umma_desc(st, P.plane, kTmHX * 16);
                    const uint64_t db0 = umma_desc(st + 2 * P.plane, 128, 256);
                    for (int j = 0; j < P.bz; ++j) {
                        // descriptor start addresses advance in 16-byte units (no carry: shared memory < 256 KB)
                        const uint64_t daj = da0 + (uint64_t)(j * kTmHY * kTmHX);
#pragma unroll
                        for (int tap = 0; tap < 27; ++tap) {
                            const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
                            tm_mma(d0 + (uint32_t)(j * BN), daj + (uint64_t)((dz * kTmHY + dy) * kTmHX + dx),
                                   db0 + (uint64_t)(tap * 2 * BN), idesc, (g > 0 || tap > 0) ? 1u : 0u);
                        }
                    }
                    tm_commit(smem_u32(&empty[s]));
                }
                if (!ok) {
                    *abort_flag = 1;
                    break;
                }
                tm_commit(smem_u32(&acc_full[a]));
            }
            // every MMA issued has completed before tensor memory is freed
            tm_commit(smem_u32(&drained));
            mbar_wait(smem_u32(&drained), 0);
        }
    } else {
        // epilogue warps 0-3
        int it = 0;
        for (int t = blockIdx.x; t < P.tiles; t += gridDim.x, ++it) {
            const int a = it & 1;
            const bool ok = !*abort_flag && tm_wait(smem_u32(&acc_full[a]), (uint32_t)((it >> 1) & 1), abort_flag);
            if (!__all_sync(0xffffffffu, ok)) {
                *abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            tm_epilogue<BN>(P, tm_tile(P, t), tmem + (uint32_t)a * acc_cols, warp, lane);
            asm volatile("tcgen05.fence::before_thread_sync;");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[a])) : "memory");
        }
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (tid == 0 && abort_word) atomicAdd(&g_conv_timeouts, 1);
    if (warp == 5)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(P.cols));
}

// ------------------------------- narrow per-voxel convolutions (CUDA cores)
// 1^3 convolutions and transposed 2^3 stride-2 convolutions with 8 or 16
// output channels: each output voxel is one dot product of its input (parent)
// voxel's channels with the weights of its tap, and a tensor-core tile of 128
// voxels x 16 channels would be mostly idle. A thread computes one output
// voxel: the input channels in 16-byte groups, the weights of all taps as FP32
// in shared memory, FP32 fused multiply-adds in channel order, then the bias,
// ReLU, accumulation and BF16 / FP32 stores of the implicit-GEMM epilogue.
constexpr int kDirectThreads = 256;
constexpr int kDirectMaxWeights = 12288;   // taps x cin x cout FP32 values (48 KB)

template <int COUT>
__global__ void __launch_bounds__(kDirectThreads) conv_direct_kernel(const __grid_constant__ Conv a) {
    extern __shared__ float ws[];          // [taps][cin][COUT]
    const int taps = a.transposed ? 8 : 1;
    const int nw = taps * a.cin * COUT;
    for (int i = threadIdx.x; i < nw; i += kDirectThreads) ws[i] = __bfloat162float(a.w[i]);
    __syncthreads();
    const long long o = (long long)blockIdx.x * kDirectThreads + threadIdx.x;
    if (o >= (long long)a.batch * a.od * a.oh * a.ow) return;
    const RowPos p = decode(o, a.od, a.oh, a.ow);
    int tap = 0;
    long long q = o;
    if (a.transposed) {
        // output voxel 2 q + j is tap j of input voxel q
        tap = ((p.z & 1) << 2) | ((p.y & 1) << 1) | (p.x & 1);
        q = (((long long)p.b * a.id + (p.z >> 1)) * a.ih + (p.y >> 1)) * a.iw + (p.x >> 1);
    }
    const float* W = ws + tap * a.cin * COUT;
    const bf16* x = a.in1.p + q * a.in1.pitch + a.in1.offset;
    float acc[COUT];
#pragma unroll
    for (int n = 0; n < COUT; ++n) acc[n] = 0.f;
    for (int c8 = 0; c8 < a.cin; c8 += 8) {
        const uint4 raw = *reinterpret_cast<const uint4*>(x + c8);
        const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&raw);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 f = __bfloat1622float2(h[e]);
            const float* w0 = W + (c8 + 2 * e) * COUT;
#pragma unroll
            for (int n = 0; n < COUT; ++n) acc[n] = __fmaf_rn(f.x, w0[n], acc[n]);
#pragma unroll
            for (int n = 0; n < COUT; ++n) acc[n] = __fmaf_rn(f.y, w0[COUT + n], acc[n]);
        }
    }
#pragma unroll
    for (int n = 0; n < COUT; ++n) {
        if (a.bias) acc[n] += __ldg(a.bias + n);
        if (a.relu) acc[n] = fmaxf(acc[n], 0.f);
    }
    if (a.out) {
        uint4* dst = reinterpret_cast<uint4*>(a.out + o * a.out_pitch + a.out_offset);
#pragma unroll
        for (int g = 0; g < COUT / 8; ++g) {
            if (a.accumulate) {
                const uint4 prev = dst[g];
                const __nv_bfloat162* pv = reinterpret_cast<const __nv_bfloat162*>(&prev);
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const float2 f = __bfloat1622float2(pv[e]);
                    acc[8 * g + 2 * e] += f.x;
                    acc[8 * g + 2 * e + 1] += f.y;
                }
            }
            uint4 pk;
            __nv_bfloat162* pp = reinterpret_cast<__nv_bfloat162*>(&pk);
#pragma unroll
            for (int e = 0; e < 4; ++e) pp[e] = __floats2bfloat162_rn(acc[8 * g + 2 * e], acc[8 * g + 2 * e + 1]);
            dst[g] = pk;
        }
    }
    if (a.out_f32) {
        float* dst = a.out_f32 + o * a.out_f32_pitch;
#pragma unroll
        for (int n = 0; n < COUT; ++n) dst[n] = acc[n];
    }
}

// Packed weights of the TMA convolution: w[k = tap * cin + c][cout] ->
// [cout / BN][groups][27][BN / 8][16][8] (channels >= cin zero), the
// MN-major core-matrix image a stage copies into shared memory as it is.
__global__ void conv3_pack_kernel(const bf16* __restrict__ w, int cin, int cout, int bn, int groups,
                                  bf16* __restrict__ packed) {
    const long long n = (long long)(cout / bn) * groups * 27 * bn * 16;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int e = (int)(i % 8);
    long long r = i / 8;
    const int row = (int)(r % 16);
    r /= 16;
    const int j = (int)(r % (bn / 8));
    r /= bn / 8;
    const int tap = (int)(r % 27);
    r /= 27;
    const int g = (int)(r % groups);
    const int nb = (int)(r / groups);
    const int c = 16 * g + row, co = nb * bn + 8 * j + e;
    packed[i] = c < cin ? w[((long long)tap * cin + c) * cout + co] : __float2bfloat16(0.f);
}

// ------------------------------------------------------ weight gradient GEMM
// dW[k][n] += sum over the block's voxel chunk of A[m][k] G[m][n]; A^T
// fragments come from the [m][k] tile through ldmatrix.trans.
__global__ void __launch_bounds__(kGemmThreads) conv_wgrad_kernel(const __grid_constant__ Conv a, const bf16* g,
                                                                 int g_pitch, float* dw, long long chunk) {
    __shared__ __align__(128) bf16 sA[kStages][16 * kWStride];
    __shared__ __align__(128) bf16 sG[kStages][16 * kBStride];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int k0 = blockIdx.x * 128, n0 = blockIdx.y * kBN;
    const int cls = a.transposed ? (int)(blockIdx.z % 8) : 0;
    const long long split = a.transposed ? blockIdx.z / 8 : blockIdx.z;
    const long long mb = split * chunk;
    const long long me = min(a.rows, mb + chunk);
    const int nsteps = (int)((me - mb + 15) / 16);
    const int u0 = k0 / 8;

    auto load = [&](int stage, int step) {
        const int ml = tid >> 3;
        const long long m = mb + (long long)step * 16 + ml;
        const bool row_ok = m < me;
        RowPos pos = {0, 0, 0, 0};
        if (row_ok) pos = a.transposed ? decode(m, a.id, a.ih, a.iw) : decode(m, a.od, a.oh, a.ow);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int ul = (tid & 7) * 2 + h;
            const int u = u0 + ul;
            const bf16* src = (row_ok && u < a.k_units) ? gather(a, pos, u) : nullptr;
            cp_async16(&sA[stage][ml * kWStride + ul * 8], src ? src : a.in1.p, src != nullptr);
        }
        const int nu = (tid & 7) * 8, n = n0 + nu;
        const bool ok = row_ok && n < a.cout;
        const bf16* src = ok ? g + out_voxel(a, m, cls) * g_pitch + n : g;
        cp_async16(&sG[stage][ml * kBStride + nu], src, ok);
    };

    float acc[2][8][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < nsteps) load(s, s);
        cp_async_commit();
    }
    for (int step = 0; step < nsteps; ++step) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        const int pf = step + kStages - 1;
        if (pf < nsteps) load(pf % kStages, pf);
        cp_async_commit();
        const int st = step % kStages;
        unsigned af[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int kt = warp * 2 + mt;
            ldmatrix_x4_trans(af[mt], &sA[st][((lane & 7) + ((lane >> 4) << 3)) * kWStride + kt * 16 +
                                              ((lane >> 3) & 1) * 8]);
        }
#pragma unroll
        for (int np = 0; np < 4; ++np) {
            unsigned bf[4];
            ldmatrix_x4_trans(bf, &sG[st][((lane & 7) + ((lane >> 3) & 1) * 8) * kBStride + np * 16 + (lane >> 4) * 8]);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                mma_bf16(acc[mt][2 * np], af[mt], bf[0], bf[1]);
                mma_bf16(acc[mt][2 * np + 1], af[mt], bf[2], bf[3]);
            }
        }
    }
    cp_async_wait<0>();
    const int k_elems = a.k_units * 8;
    float* base = dw + (a.transposed ? (size_t)cls * a.cin * a.cout : 0);
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int k = k0 + warp * 32 + mt * 16 + (lane >> 2) + half * 8;
            if (k >= k_elems) continue;
#pragma unroll
            for (int nt = 0; nt < 8; ++nt) {
                const int n = n0 + nt * 8 + (lane & 3) * 2;
                if (n >= a.cout) continue;
                atomicAdd(base + (size_t)k * a.cout + n, acc[mt][nt][half * 2]);
                atomicAdd(base + (size_t)k * a.cout + n + 1, acc[mt][nt][half * 2 + 1]);
            }
        }
}

// ------------------------------------------------------------ elementwise
// dy *= (y > 0): the ReLU derivative, in place.
__global__ void relu_backward_kernel(long long voxels, int channels, bf16* dy, int dy_pitch, const bf16* y,
                                     int y_pitch, int y_offset) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= voxels * channels) return;
    const long long v = i / channels;
    const int c = (int)(i - v * channels);
    if (!(__bfloat162float(y[v * y_pitch + y_offset + c]) > 0.f)) dy[v * dy_pitch + c] = __float2bfloat16_rn(0.f);
}

// db[c] += sum over voxels of g[v][c] (block-local FP32 sums, one atomic per channel and block).
__global__ void bias_grad_kernel(long long voxels, int channels, const bf16* g, int pitch, float* db) {
    __shared__ float part[128];
    for (int c = threadIdx.x; c < channels; c += blockDim.x) part[c] = 0.f;
    __syncthreads();
    const long long per = (voxels + gridDim.x - 1) / gridDim.x;
    const long long vb = blockIdx.x * per, ve = min(voxels, vb + per);
    for (int c = threadIdx.x % channels; c < channels; c += channels) {
        float s = 0.f;
        for (long long v = vb + threadIdx.x / channels; v < ve; v += blockDim.x / channels)
            s += __bfloat162float(g[v * pitch + c]);
        atomicAdd(&part[c], s);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < channels; c += blockDim.x) atomicAdd(db + c, part[c]);
}

// Adam on FP32 master weights, refreshing their BF16 copy.
__global__ void adam_kernel(long long n, float* w, float* m, float* v, const float* g, bf16* w16, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16_rn(wi);
}

// Network input: channel 0 = scale * divergence, channel 1 = solid mask,
// channels 2..7 = 0 (the first convolution reads 8 channels).
// out = src * scale; with `max_abs`, scale = 1 / (input_scale * weight) in
// FP64 (0 for a zero input), the factor that undoes the input normalisation.
__global__ void unpack_channel_kernel(long long voxels, const float* __restrict__ src, int pitch, float scale,
                                      const float* max_abs, double weight, float* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (max_abs) {
        const float m = *max_abs;
        scale = m > 0.f ? (float)(1.0 / ((1.0 / (double)m) * weight)) : 0.f;
    }
    if (i < voxels) out[i] = src[i * pitch] * scale;
}

// Coarse collider mask: a coarse cell is solid when at least `threshold` of its
// eight children are.
__global__ void mask_restrict_kernel(int cx, int cy, int cz, const uint8_t* __restrict__ fine, int threshold,
                                     uint8_t* __restrict__ coarse) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= (long long)cx * cy * cz) return;
    const int x = (int)(c % cx), y = (int)((c / cx) % cy), z = (int)(c / ((long long)cx * cy));
    const int fx = 2 * cx, fy = 2 * cy;
    int n = 0;
    for (int dz = 0; dz < 2; ++dz)
        for (int dy = 0; dy < 2; ++dy)
            for (int dx = 0; dx < 2; ++dx)
                n += fine[(2 * x + dx) + (long long)fx * ((2 * y + dy) + (long long)fy * (2 * z + dz))] != 0;
    coarse[c] = n >= threshold ? 1 : 0;
}

// Scale of the network's input from max |div| on the device: 1 / max (0 when
// the field is zero), the FP32 rounding of the FP64 quotient, as a host would
// form it.
__device__ __forceinline__ float input_scale(const float* max_abs) {
    const float m = *max_abs;
    return m > 0.f ? (float)(1.0 / (double)m) : 0.f;
}

__global__ void pack_input_kernel(long long voxels, const float* div, const uint8_t* mask, float scale,
                                  const float* max_abs, bf16* out) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= voxels) return;
    if (max_abs) scale = input_scale(max_abs);
    __align__(16) bf16 c[8];
    c[0] = __float2bfloat16_rn(scale * div[v]);
    c[1] = __float2bfloat16_rn(mask && mask[v] ? 1.f : 0.f);
#pragma unroll
    for (int k = 2; k < 8; ++k) c[k] = __float2bfloat16_rn(0.f);
    *reinterpret_cast<uint4*>(out + v * 8) = *reinterpret_cast<const uint4*>(c);
}

// Loss sum_v (pred - target)^2 / count over fluid voxels and its gradient,
// written into channel 0 of an 8-channel BF16 tensor (the head's input gradient
// is formed from it by the head's data-gradient convolution).
__global__ void mse_kernel(long long voxels, const float* pred, int pred_pitch, const float* target,
                           const uint8_t* mask, float inv_count, bf16* grad, double* loss) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (v < voxels) {
        const bool fluid = !(mask && mask[v]);
        const float d = fluid ? pred[v * pred_pitch] - target[v] : 0.f;
        e = (double)d * d * inv_count;
        __align__(16) bf16 c[8];
        c[0] = __float2bfloat16_rn(2.f * d * inv_count);
#pragma unroll
        for (int k = 1; k < 8; ++k) c[k] = __float2bfloat16_rn(0.f);
        *reinterpret_cast<uint4*>(grad + v * 8) = *reinterpret_cast<const uint4*>(c);
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0 && e != 0.0) atomicAdd(loss, e);
}

// dst[t][co][ci] = src[flip ? taps - 1 - t : t][ci][co]: the weights of the
// data-gradient convolution (transposed per tap; taps reversed for a padded
// convolution whose gradient correlates with the mirrored kernel).
__global__ void weight_transpose_kernel(int taps, int cin, int cout, int flip, const bf16* src, bf16* dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long n = (long long)taps * cin * cout;
    if (i >= n) return;
    const int ci = (int)(i % cin);
    const long long r = i / cin;
    const int co = (int)(r % cout);
    const int t = (int)(r / cout);
    const int ts = flip ? taps - 1 - t : t;
    dst[i] = src[((long long)ts * cin + ci) * cout + co];
}

bool view_ok(const FfxTensorView& t, int channels) {
    return t.data && t.pitch >= t.offset + channels && t.pitch % 8 == 0 && t.offset % 8 == 0 &&
           ((uintptr_t)t.data & 15) == 0;
}

int make_conv(const FfxConv* c, Conv& a) {
    FFX_REQUIRE(c && c->batch >= 1 && c->c1 >= 8 && c->c1 % 8 == 0 && c->c2 >= 0 && c->c2 % 8 == 0 &&
                    c->cout >= 8 && c->cout % 8 == 0 && c->weight && ((uintptr_t)c->weight & 15) == 0,
                "ffx_conv: invalid arguments (channels multiples of 8, 16-byte aligned weights)");
    for (int i = 0; i < 3; ++i)
        FFX_REQUIRE(c->in_dims[i] >= 1 && c->out_dims[i] >= 1 && c->in_dims[i] <= 4096 && c->out_dims[i] <= 4096,
                    "ffx_conv: invalid dimensions");
    FFX_REQUIRE(view_ok(c->in1, c->c1) && (c->c2 == 0 || view_ok(c->in2, c->c2)),
                "ffx_conv: input views need 16-byte aligned data, pitch and offset multiples of 8");
    if (c->transposed) {
        FFX_REQUIRE(c->ksize == 2 && c->stride == 2 && c->pad == 0 && c->out_dims[0] == 2 * c->in_dims[0] &&
                        c->out_dims[1] == 2 * c->in_dims[1] && c->out_dims[2] == 2 * c->in_dims[2],
                    "ffx_conv: the transposed form is 2^3 with stride 2 onto a grid twice as large");
    } else {
        FFX_REQUIRE(c->ksize >= 1 && c->ksize <= 3 && c->stride >= 1 && c->stride <= 2 && c->pad >= 0 &&
                        c->pad < c->ksize,
                    "ffx_conv: kernel size 1..3, stride 1..2, pad < kernel size");
        for (int i = 0; i < 3; ++i)
            FFX_REQUIRE(c->out_dims[i] == (c->in_dims[i] + 2 * c->pad - c->ksize) / c->stride + 1,
                        "ffx_conv: output dimensions do not follow from input, kernel, stride and pad");
    }
    if (c->out)
        FFX_REQUIRE(c->out_pitch >= c->out_offset + c->cout && c->out_pitch % 8 == 0 && c->out_offset % 8 == 0 &&
                        ((uintptr_t)c->out & 15) == 0,
                    "ffx_conv: output view");
    if (c->out_f32) FFX_REQUIRE(c->out_f32_pitch >= c->cout && c->out_f32_pitch % 2 == 0, "ffx_conv: FP32 output pitch");
    a.batch = c->batch;
    a.id = c->in_dims[0]; a.ih = c->in_dims[1]; a.iw = c->in_dims[2];
    a.od = c->out_dims[0]; a.oh = c->out_dims[1]; a.ow = c->out_dims[2];
    a.c1 = c->c1; a.c2 = c->c2; a.cin = c->c1 + c->c2; a.cout = c->cout;
    a.ks = c->ksize; a.stride = c->stride; a.pad = c->pad; a.transposed = c->transposed;
    a.taps = c->transposed ? 1 : c->ksize * c->ksize * c->ksize;
    a.units_per_tap = a.cin / 8;
    a.k_units = a.taps * a.units_per_tap;
    const long long in_vox = (long long)a.batch * a.id * a.ih * a.iw;
    a.rows = c->transposed ? in_vox : (long long)a.batch * a.od * a.oh * a.ow;
    FFX_REQUIRE(a.rows < (1LL << 40), "ffx_conv: too many voxels");
    a.in1 = View{(const bf16*)c->in1.data, c->in1.pitch, c->in1.offset};
    a.in2 = View{(const bf16*)(c->c2 ? c->in2.data : c->in1.data), c->c2 ? c->in2.pitch : 8,
                 c->c2 ? c->in2.offset : 0};
    a.w = (const bf16*)c->weight;
    a.bias = c->bias;
    a.relu = c->relu;
    a.accumulate = c->accumulate;
    a.out = (bf16*)c->out;
    a.out_pitch = c->out_pitch;
    a.out_offset = c->out_offset;
    a.out_f32 = c->out_f32;
    a.out_f32_pitch = c->out_f32_pitch;
    return FFX_OK;
}

// ---------------------------------------------- TMA convolution, host side
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled from the driver the runtime loaded (no link-time libcuda).
EncodeTiled tensor_map_encoder() {
    static EncodeTiled fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    }
    return fn;
}

// 3x3x3, stride 1, pad 1, one input view, channels the kernel tiles.
bool tma_eligible(const Conv& a) {
    return !a.transposed && a.ks == 3 && a.stride == 1 && a.pad == 1 && a.c2 == 0 &&
           (a.cin % 16 == 0 || a.cin == 8) && a.cin <= 512 && a.cout % 16 == 0 && a.od == a.id && a.oh == a.ih &&
           a.ow == a.iw;
}
int tma_bn(int cout) { return cout % 64 == 0 ? 64 : (cout % 32 == 0 ? 32 : 16); }
int tma_groups(int cin) { return (cin + 15) / 16; }
long long tma_packed_elems(const Conv& a) { return (long long)tma_groups(a.cin) * 27 * 16 * a.cout; }

int sm_count() {
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) !=
                                                     cudaSuccess || n <= 0)
            n = 148;
    }
    return n;
}

}  // namespace
}  // namespace ffx

using namespace ffx;

extern "C" {

int ffx_conv_forward(const FfxConv* c, void* stream) {
    Conv a;
    int e = make_conv(c, a);
    if (e) return e;
    FFX_REQUIRE(a.out || a.out_f32, "ffx_conv_forward: no output");
    const int bn = a.cout <= 16 ? 16 : (a.cout <= 32 ? 32 : 64);
    const dim3 grid((unsigned)((a.rows + kBM - 1) / kBM), (unsigned)((a.cout + bn - 1) / bn), a.transposed ? 8 : 1);
    FFX_REQUIRE(grid.x < (1u << 31), "ffx_conv_forward: grid too large");
    if (bn == 16) conv_fwd_kernel<16><<<grid, kGemmThreads, 0, as_stream(stream)>>>(a);
    else if (bn == 32) conv_fwd_kernel<32><<<grid, kGemmThreads, 0, as_stream(stream)>>>(a);
    else conv_fwd_kernel<64><<<grid, kGemmThreads, 0, as_stream(stream)>>>(a);
    return launch_status("conv_fwd_kernel");
}

int ffx_conv_forward_tc(const FfxConv* c, void* stream) {
    Conv a;
    int e = make_conv(c, a);
    if (e) return e;
    FFX_REQUIRE(a.out || a.out_f32, "ffx_conv_forward_tc: no output");
    const int bn = a.cout <= 16 ? 16 : (a.cout <= 32 ? 32 : 64);
    const dim3 grid((unsigned)((a.rows + kBM - 1) / kBM), (unsigned)((a.cout + bn - 1) / bn), a.transposed ? 8 : 1);
    FFX_REQUIRE(grid.x < (1u << 31), "ffx_conv_forward_tc: grid too large");
    static bool configured = false;     // dynamic shared memory above 48 KB, once per process
    if (!configured) {
        cudaFuncSetAttribute(conv_fwd_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<16>());
        cudaFuncSetAttribute(conv_fwd_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<32>());
        cudaFuncSetAttribute(conv_fwd_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes<64>());
        configured = true;
    }
    cudaStream_t st = as_stream(stream);
    if (bn == 16) conv_fwd_tc_kernel<16><<<grid, kGemmThreads, tc_smem_bytes<16>(), st>>>(a);
    else if (bn == 32) conv_fwd_tc_kernel<32><<<grid, kGemmThreads, tc_smem_bytes<32>(), st>>>(a);
    else conv_fwd_tc_kernel<64><<<grid, kGemmThreads, tc_smem_bytes<64>(), st>>>(a);
    return launch_status("conv_fwd_tc_kernel");
}

int ffx_conv_packed_bytes(const FfxConv* c, int64_t* bytes) {
    FFX_REQUIRE(bytes, "ffx_conv_packed_bytes: invalid arguments");
    Conv a;
    int e = make_conv(c, a);
    if (e) return e;
    *bytes = tma_eligible(a) ? tma_packed_elems(a) * 2 : 0;
    return FFX_OK;
}

int ffx_conv_pack_weights(const FfxConv* c, void* packed, void* stream) {
    Conv a;
    int e = make_conv(c, a);
    if (e) return e;
    FFX_REQUIRE(tma_eligible(a), "ffx_conv_pack_weights: not a 3x3x3 stride-1 pad-1 convolution the TMA kernel tiles");
    FFX_REQUIRE(packed && ((uintptr_t)packed & 15) == 0, "ffx_conv_pack_weights: packed buffer (16-byte aligned)");
    const long long n = tma_packed_elems(a);
    conv3_pack_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(a.w, a.cin, a.cout, tma_bn(a.cout),
                                                                        tma_groups(a.cin), (bf16*)packed);
    return launch_status("conv3_pack_kernel");
}

int ffx_conv_forward_tma(const FfxConv* c, const void* packed, void* stream) {
    Conv a;
    int e = make_conv(c, a);
    if (e) return e;
    if (!tma_eligible(a)) {
        // 1^3 and transposed 2^3 layers with 8 or 16 output channels: the per-voxel kernel;
        // the remaining shapes: the mma.sync implicit GEMM
        const bool one = !a.transposed && a.ks == 1 && a.stride == 1 && a.pad == 0;
        if ((one || a.transposed) && (a.cout == 8 || a.cout == 16) && a.c2 == 0 &&
            (a.transposed ? 8 : 1) * a.cin * a.cout <= kDirectMaxWeights && (a.out || a.out_f32)) {
            const long long vox = (long long)a.batch * a.od * a.oh * a.ow;
            const size_t smem = sizeof(float) * (size_t)(a.transposed ? 8 : 1) * a.cin * a.cout;
            const unsigned blocks = (unsigned)((vox + kDirectThreads - 1) / kDirectThreads);
            if (a.cout == 8) conv_direct_kernel<8><<<blocks, kDirectThreads, smem, as_stream(stream)>>>(a);
            else conv_direct_kernel<16><<<blocks, kDirectThreads, smem, as_stream(stream)>>>(a);
            return launch_status("conv_direct_kernel");
        }
        return ffx_conv_forward(c, stream);
    }
    FFX_REQUIRE(a.out || a.out_f32, "ffx_conv_forward_tma: no output");
    FFX_REQUIRE(packed && ((uintptr_t)packed & 15) == 0,
                "ffx_conv_forward_tma: packed weights (ffx_conv_pack_weights, 16-byte aligned)");
    FFX_REQUIRE(!a.out_f32 || a.out_f32_pitch >= a.cout, "ffx_conv_forward_tma: FP32 output pitch");
    EncodeTiled encode = tensor_map_encoder();
    FFX_REQUIRE(encode, "ffx_conv_forward_tma: cuTensorMapEncodeTiled is not available from the driver");
    const int bn = tma_bn(a.cout);
    TmaConv P;
    std::memset(&P, 0, sizeof(P));
    P.wpack = (const bf16*)packed;
    P.batch = a.batch;
    P.d = a.id; P.h = a.ih; P.w = a.iw;
    P.cin = a.cin; P.cout = a.cout; P.groups = tma_groups(a.cin);
    P.planes = a.cin == 8 ? 1 : 2;
    P.tiles_x = (a.iw + kTmX - 1) / kTmX;
    P.tiles_y = (a.ih + kTmY - 1) / kTmY;
    // deepest tile (z slices sharing one halo) that still gives every SM two tiles
    const long long nblocks = a.cout / bn;
    const long long want = 2LL * sm_count();
    P.bz = 1;
    for (int bz = 4; bz >= 1; bz >>= 1) {
        const long long blocks = (long long)P.tiles_x * P.tiles_y * ((a.id + bz - 1) / bz) * a.batch * nblocks;
        if (blocks >= want || bz == 1) { P.bz = bz; break; }
    }
    P.tiles_z = (a.id + P.bz - 1) / P.bz;
    P.nblocks = (int)nblocks;
    const long long tiles = (long long)P.tiles_x * P.tiles_y * P.tiles_z * a.batch * nblocks;
    FFX_REQUIRE(tiles < (1LL << 31), "ffx_conv_forward_tma: too many tiles");
    P.tiles = (int)tiles;
    const uint32_t box_bytes = 8u * kTmHX * kTmHY * (uint32_t)(P.bz + 2) * 2u;
    P.plane = (box_bytes + 127u) & ~127u;
    P.stage = 2 * P.plane + 27u * 32u * (uint32_t)bn;
    P.tx = (uint32_t)P.planes * box_bytes + 27u * 32u * (uint32_t)bn;
    // as many stages as fit (the ring runs across tiles), at most four
    P.stages = std::min(kTmMaxStages, (int)((kTmSmemLimit - 128u) / P.stage));
    FFX_REQUIRE(P.stages >= 1, "ffx_conv_forward_tma: a stage does not fit in shared memory");
    const size_t smem = (size_t)P.stages * P.stage + 128;
    const uint32_t need = 2u * (uint32_t)P.bz * (uint32_t)bn;    // two accumulator sets
    P.cols = need <= 32 ? 32u : (need <= 64 ? 64u : (need <= 128 ? 128u : (need <= 256 ? 256u : 512u)));
    FFX_REQUIRE(need <= 512, "ffx_conv_forward_tma: accumulators exceed tensor memory");
    // persistent: one block per SM (the stage ring fills its shared memory)
    const long long blocks = std::min<long long>(tiles, sm_count());
    P.bias = a.bias;
    P.relu = a.relu;
    P.accumulate = a.accumulate;
    P.out = a.out;
    P.out_pitch = a.out_pitch;
    P.out_offset = a.out_offset;
    P.out_f32 = a.out_f32;
    P.out_f32_pitch = a.out_f32_pitch;
    // input activations as a (channel, x, y, z, batch) tensor, zero outside
    const cuuint64_t pitch = (cuuint64_t)a.in1.pitch * 2;
    const cuuint64_t dims[5] = {(cuuint64_t)a.cin, (cuuint64_t)a.iw, (cuuint64_t)a.ih, (cuuint64_t)a.id,
                                (cuuint64_t)a.batch};
    const cuuint64_t strides[4] = {pitch, pitch * a.iw, pitch * a.iw * a.ih, pitch * a.iw * a.ih * a.id};
    const cuuint32_t box[5] = {8, kTmHX, kTmHY, (cuuint32_t)(P.bz + 2), 1};
    const cuuint32_t estride[5] = {1, 1, 1, 1, 1};
    const CUresult r = encode(&P.act, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, (void*)(a.in1.p + a.in1.offset), dims,
                              strides, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    FFX_REQUIRE(r == CUDA_SUCCESS, "ffx_conv_forward_tma: cuTensorMapEncodeTiled rejected the input view");
    static bool configured = false;
    if (!configured) {
        cudaFuncSetAttribute(conv3_tma_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmSmemLimit);
        cudaFuncSetAttribute(conv3_tma_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmSmemLimit);
        cudaFuncSetAttribute(conv3_tma_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTmSmemLimit);
        configured = true;
    }
    const dim3 grid((unsigned)blocks, 1, 1);
    cudaStream_t st = as_stream(stream);
    if (bn == 16) conv3_tma_kernel<16><<<grid, kTmThreads, smem, st>>>(P);
    else if (bn == 32) conv3_tma_kernel<32><<<grid, kTmThreads, smem, st>>>(P);
    else conv3_tma_kernel<64><<<grid, kTmThreads, smem, st>>>(P);
    return launch_status("conv3_tma_kernel");
}

int ffx_conv_timeouts(int32_t* out, int32_t reset) {
    FFX_REQUIRE(out, "ffx_conv_timeouts: invalid arguments");
    int e = cuda_status(cudaMemcpyFromSymbol(out, g_conv_timeouts, sizeof(int32_t)), "ffx_conv_timeouts: read");
    if (e) return e;
    if (reset) {
        const int32_t zero = 0;
        e = cuda_status(cudaMemcpyToSymbol(g_conv_timeouts, &zero, sizeof(int32_t)), "ffx_conv_timeouts: reset");
    }
    return e;
}

int ffx_conv_weight_grad(const FfxConv* c, const void* grad, int32_t grad_pitch, float* dweight, void* stream) {
    Conv a;
    int e = make_conv(c, a);
    if (e) return e;
    FFX_REQUIRE(grad && dweight && grad_pitch >= c->cout && grad_pitch % 8 == 0 && ((uintptr_t)grad & 15) == 0,
                "ffx_conv_weight_grad: invalid gradient view");
    const long long chunk = 8192;
    const long long splits = (a.rows + chunk - 1) / chunk;
    FFX_REQUIRE(splits * (a.transposed ? 8 : 1) < 65536, "ffx_conv_weight_grad: too many voxels for one launch");
    const dim3 grid((unsigned)((a.k_units * 8 + 127) / 128), (unsigned)((a.cout + kBN - 1) / kBN),
                    (unsigned)(splits * (a.transposed ? 8 : 1)));
    conv_wgrad_kernel<<<grid, kGemmThreads, 0, as_stream(stream)>>>(a, (const bf16*)grad, grad_pitch, dweight, chunk);
    return launch_status("conv_wgrad_kernel");
}

int ffx_relu_backward(int64_t voxels, int32_t channels, void* dy, int32_t dy_pitch, const void* y, int32_t y_pitch,
                      int32_t y_offset, void* stream) {
    FFX_REQUIRE(voxels >= 1 && channels >= 1 && dy && y && dy_pitch >= channels && y_pitch >= y_offset + channels,
                "ffx_relu_backward: invalid arguments");
    const long long n = voxels * channels;
    relu_backward_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(voxels, channels, (bf16*)dy, dy_pitch,
                                                                             (const bf16*)y, y_pitch, y_offset);
    return launch_status("relu_backward_kernel");
}

int ffx_bias_grad(int64_t voxels, int32_t channels, const void* g, int32_t pitch, float* dbias, void* stream) {
    FFX_REQUIRE(voxels >= 1 && channels >= 1 && channels <= 128 && 256 % channels == 0 && g && dbias &&
                    pitch >= channels,
                "ffx_bias_grad: invalid arguments (channels divide 256, at most 128)");
    const long long blocks = std::min<long long>(1184, (voxels + 255) / 256);
    bias_grad_kernel<<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(voxels, channels, (const bf16*)g, pitch, dbias);
    return launch_status("bias_grad_kernel");
}

int ffx_adam(int64_t n, float* w, float* m, float* v, const float* g, void* w_bf16, float lr, float beta1,
             float beta2, float eps, int32_t step, void* stream) {
    FFX_REQUIRE(n >= 1 && w && m && v && g && step >= 1 && lr > 0.f, "ffx_adam: invalid arguments");
    const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
    adam_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(n, w, m, v, g, (bf16*)w_bf16, lr, beta1, beta2,
                                                                    eps, c1, c2);
    return launch_status("adam_kernel");
}

int ffx_weight_transpose(int32_t taps, int32_t cin, int32_t cout, int32_t flip, const void* src, void* dst,
                         void* stream) {
    FFX_REQUIRE(taps >= 1 && cin >= 1 && cout >= 1 && src && dst && src != dst, "ffx_weight_transpose: invalid arguments");
    const long long n = (long long)taps * cin * cout;
    weight_transpose_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(taps, cin, cout, flip, (const bf16*)src,
                                                                                (bf16*)dst);
    return launch_status("weight_transpose_kernel");
}

int ffx_pack_input(int64_t voxels, const float* div, const uint8_t* mask, float scale, void* out, void* stream) {
    FFX_REQUIRE(voxels >= 1 && div && out && ((uintptr_t)out & 15) == 0, "ffx_pack_input: invalid arguments");
    pack_input_kernel<<<blocks_for(voxels, 256), 256, 0, as_stream(stream)>>>(voxels, div, mask, scale, nullptr,
                                                                            (bf16*)out);
    return launch_status("pack_input_kernel");
}

int ffx_pack_input_scaled(int64_t voxels, const float* div, const uint8_t* mask, const float* max_abs, void* out,
                          void* stream) {
    FFX_REQUIRE(voxels >= 1 && div && max_abs && out && ((uintptr_t)out & 15) == 0,
                "ffx_pack_input_scaled: invalid arguments");
    pack_input_kernel<<<blocks_for(voxels, 256), 256, 0, as_stream(stream)>>>(voxels, div, mask, 0.f, max_abs,
                                                                            (bf16*)out);
    return launch_status("pack_input_kernel");
}

int ffx_mask_restrict(const int32_t coarse_n[3], const uint8_t* fine, int32_t threshold, uint8_t* coarse,
                      void* stream) {
    FFX_REQUIRE(coarse_n && coarse_n[0] >= 1 && coarse_n[1] >= 1 && coarse_n[2] >= 1 && fine && coarse &&
                threshold >= 1 && threshold <= 8 &&
                (int64_t)coarse_n[0] * coarse_n[1] * coarse_n[2] * 8 < (int64_t(1) << 40),
                "ffx_mask_restrict: invalid arguments");
    const int64_t n = (int64_t)coarse_n[0] * coarse_n[1] * coarse_n[2];
    mask_restrict_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(coarse_n[0], coarse_n[1], coarse_n[2],
                                                                            fine, threshold, coarse);
    return launch_status("mask_restrict_kernel");
}

int ffx_unpack_channel(int64_t voxels, const float* src, int32_t pitch, float scale, float* out, void* stream) {
    FFX_REQUIRE(voxels >= 1 && src && out && pitch >= 1, "ffx_unpack_channel: invalid arguments");
    unpack_channel_kernel<<<blocks_for(voxels, 256), 256, 0, as_stream(stream)>>>(voxels, src, pitch, scale, nullptr,
                                                                                0.0, out);
    return launch_status("unpack_channel_kernel");
}

int ffx_unpack_channel_scaled(int64_t voxels, const float* src, int32_t pitch, const float* max_abs, double weight,
                              float* out, void* stream) {
    FFX_REQUIRE(voxels >= 1 && src && max_abs && out && pitch >= 1, "ffx_unpack_channel_scaled: invalid arguments");
    unpack_channel_kernel<<<blocks_for(voxels, 256), 256, 0, as_stream(stream)>>>(voxels, src, pitch, 0.f, max_abs,
                                                                                weight, out);
    return launch_status("unpack_channel_kernel");
}

int ffx_mse_grad(int64_t voxels, const float* pred, int32_t pred_pitch, const float* target, const uint8_t* mask,
                 float inv_count, void* grad, double* loss, void* stream) {
    FFX_REQUIRE(voxels >= 1 && pred && target && grad && loss && pred_pitch >= 1 && ((uintptr_t)grad & 15) == 0,
                "ffx_mse_grad: invalid arguments");
    mse_kernel<<<blocks_for(voxels, 256), 256, 0, as_stream(stream)>>>(voxels, pred, pred_pitch, target, mask,
                                                                        inv_count, (bf16*)grad, loss);
    return launch_status("mse_kernel");
}

}  // extern "C"
