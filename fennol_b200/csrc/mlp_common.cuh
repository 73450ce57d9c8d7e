// Shared pieces of the species-MLP kernels.
#pragma once
#include "common.cuh"

namespace fnl {

// jax.nn.celu(x, alpha) = x if x > 0 else alpha * expm1(x / alpha)
__device__ __forceinline__ float celu_f(float x, float alpha) {
  return x > 0.f ? x : alpha * expm1f(x / alpha);
}

// celu'(z) recovered from h = celu(z): 1 for h > 0, exp(z/alpha) = h/alpha + 1 otherwise.
__device__ __forceinline__ float dcelu_from_h(float h, float alpha) {
  return h > 0.f ? 1.f : h / alpha + 1.f;
}

}  // namespace fnl

// Entry points of the individual MLP implementations (C++ linkage, internal).
size_t fnl_mlp_simt_workspace(int rows, const fennol_mlp_weights* w);
int fnl_mlp_simt(int rows, int ntiles, const int* tile_species, const int* tile_row,
                 const fennol_mlp_weights* w, const float* x, float* e_rows, float* dx, void* ws,
                 cudaStream_t st);
size_t fnl_mlp_tc_workspace(int precision, int rows, int n_models, const fennol_mlp_weights* w);
int fnl_mlp_tc(int precision, int rows, int ntiles, const int* tile_species, const int* tile_row,
               const fennol_mlp_weights* w, const void* x, const void* x_lo, unsigned long long kmask,
               float* e_rows, float* dx, void* ws, size_t ws_bytes, cudaStream_t st);
bool fnl_mlp_fused_supported(int precision, const fennol_mlp_weights* w);
size_t fnl_mlp_fused_workspace(const fennol_mlp_weights* w);
int fnl_mlp_fused(int precision, int rows, int ntiles, const int* tile_species, const int* tile_row,
                  const fennol_mlp_weights* w, const void* x, const void* x_lo, unsigned long long kmask,
                  float* e_rows, float* dx, void* ws, size_t ws_bytes, cudaStream_t st);
