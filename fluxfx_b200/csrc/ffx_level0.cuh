// Host launchers of the four-cells-per-thread level-0 kernels (ffx_level0.cu),
// used by the graph entry points when level0_x4() accepts the level and the
// float fields (link field present, nx % 4 == 0, 16-byte aligned rows).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <initializer_list>

#include "../../include/ffx.h"

namespace ffx {

bool level0_x4(const FfxGraphLevel* lv, std::initializer_list<const void*> f4);
int level0_smooth(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                  cudaStream_t st);
int level0_smooth_dot(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                      double* dot, double scale, cudaStream_t st);
int level0_smooth_zero(const FfxGraphLevel* lv, const float* rhs, float omega, float* out, cudaStream_t st);
int level0_prolong_smooth(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                          float omega, float* out, cudaStream_t st);
int level0_prolong_smooth_dot(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                              float omega, float* out, double* dot, double scale, cudaStream_t st);
int level0_smooth2(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                   cudaStream_t st);
int level0_prolong_smooth2(const FfxGraphLevel* lv, const float* p, const float* coarse, const float* rhs,
                           float omega, float* out, cudaStream_t st);
int level0_residual(const FfxGraphLevel* lv, const float* p, const float* rhs, float* r, cudaStream_t st);
int level0_residual_max(const FfxGraphLevel* lv, const float* p, const float* rhs, float* out, cudaStream_t st);
int level0_residual_max_smooth(const FfxGraphLevel* lv, const float* p, const float* rhs, float omega, float* out,
                               float* p_out, cudaStream_t st);
int level0_residual_restrict(const FfxGraphLevel* lv, const float* p, const float* rhs, float* coarse,
                             float* zero, cudaStream_t st);
int level0_direction_apply(const FfxGraphLevel* lv, const float* z, const float* p_old, const double* rz_new,
                           const double* rz_old, float* p_out, float* q, double* pq, cudaStream_t st);
int level0_links(int nx, int ny, int nz, const uint8_t* solid, uint8_t* links, cudaStream_t st);

}  // namespace ffx
