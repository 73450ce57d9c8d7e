// Shared device helpers for the fennol_b200 kernels (sm_100a).
#pragma once
#include <utility>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "fennol_b200.h"

#define FNL_WARP 32

namespace fnl {

// Device status words (int32[FENNOL_STATUS_WORDS]); the host reads them after a
// launch, like the reference's `overflow` flags (preprocessing.py:578-585).
enum StatusWord {
  ST_NBR_OVERFLOW = 0,    // a neighbour row did not fit: 1
  ST_NBR_MAXCOUNT = 1,    // largest neighbour count seen by the builder
  ST_FILTER_OVERFLOW = 2, // filtered row did not fit
  ST_FILTER_MAXCOUNT = 3, // largest filtered count
  ST_ANG_OVERFLOW = 4,    // angular neighbours beyond the in-kernel staging size
  ST_ANG_MAXCOUNT = 5,    // largest angular neighbour count
  ST_CELL_OVERFLOW = 6,   // cell list inconsistency (should never be set)
  ST_REBUILD_COUNT = 7,   // number of neighbour rebuilds executed (MD)
  ST_NONFINITE = 8,       // a checked buffer held a NaN or an infinity
};

// Packed periodic shift: three signed bytes (x | y<<8 | z<<16).
__host__ __device__ __forceinline__ unsigned pack_shift(int sx, int sy, int sz) {
  return (unsigned)(sx & 0xFF) | ((unsigned)(sy & 0xFF) << 8) | ((unsigned)(sz & 0xFF) << 16);
}
__host__ __device__ __forceinline__ void unpack_shift(unsigned s, int& sx, int& sy, int& sz) {
  sx = (int)(signed char)(s & 0xFF);
  sy = (int)(signed char)((s >> 8) & 0xFF);
  sz = (int)(signed char)((s >> 16) & 0xFF);
}

// vec += shift @ cell with a fixed order and no FMA contraction:
// component k = ((sx*c[0][k] + sy*c[1][k]) + sz*c[2][k]).  Exact for
// orthorhombic cells and |s| <= 2; matches numpy's `vec + np.dot(s, cell)`.
__device__ __forceinline__ void add_shift(float& vx, float& vy, float& vz, float sx, float sy,
                                          float sz, const float* c) {
  float tx = __fadd_rn(__fadd_rn(__fmul_rn(sx, c[0]), __fmul_rn(sy, c[3])), __fmul_rn(sz, c[6]));
  float ty = __fadd_rn(__fadd_rn(__fmul_rn(sx, c[1]), __fmul_rn(sy, c[4])), __fmul_rn(sz, c[7]));
  float tz = __fadd_rn(__fadd_rn(__fmul_rn(sx, c[2]), __fmul_rn(sy, c[5])), __fmul_rn(sz, c[8]));
  vx = __fadd_rn(vx, tx);
  vy = __fadd_rn(vy, ty);
  vz = __fadd_rn(vz, tz);
}

// (x*x + y*y) + z*z rounded like numpy's float32 `(vec**2).sum(-1)`.
__device__ __forceinline__ float dist2_exact(float vx, float vy, float vz) {
  return __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
}

// v @ recip for one column d (fixed order, no FMA).
__device__ __forceinline__ float frac_exact(float vx, float vy, float vz, const float* r, int d) {
  return __fadd_rn(__fadd_rn(__fmul_rn(vx, r[d]), __fmul_rn(vy, r[3 + d])), __fmul_rn(vz, r[6 + d]));
}

__device__ __forceinline__ void status_max(int* status, int word, int v) {
  if (status) atomicMax(status + word, v);
}
__device__ __forceinline__ void status_set(int* status, int word) {
  if (status) atomicOr(status + word, 1);
}

__device__ __forceinline__ int warp_exclusive_prefix(unsigned mask, int lane) {
  return __popc(mask & ((1u << lane) - 1u));
}

// triu index of the species pair (s1, s2) in np.triu_indices(S, 0) order.
__host__ __device__ __forceinline__ int triu_pair(int s1, int s2, int S) {
  int a = s1 < s2 ? s1 : s2, b = s1 < s2 ? s2 : s1;
  return a * S - (a * (a - 1)) / 2 + (b - a);
}

}  // namespace fnl

// Programmatic dependent launch: a kernel launched with launch_pdl may be
// scheduled while the previous kernel of the stream drains; it must call
// pdl_wait() before touching memory, which returns once that kernel has
// completed and its writes are visible (a no-op for ordinary launches).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

#define FNL_LAUNCH_PDL(...)                                      \
  do {                                                           \
    if (launch_pdl(__VA_ARGS__) != cudaSuccess) return FENNOL_ERR_CUDA; \
  } while (0)

#define FNL_CHECK_LAUNCH()                                   \
  do {                                                       \
    cudaError_t e__ = cudaGetLastError();                    \
    if (e__ != cudaSuccess) return FENNOL_ERR_CUDA;          \
  } while (0)
