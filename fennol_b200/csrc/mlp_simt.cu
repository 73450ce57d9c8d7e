// Species-indexed MLP in float32 on CUDA cores (the plain FP32 form).
//
// Replaces SpeciesIndexNet / FullyConnectedNet (src/fennol/models/misc/nets.py:
// 13-102, 301-426) and the transpose jax.grad builds for the input gradient.
// Rows are grouped by species in 128-row tiles; each tile multiplies by the
// weights of its species.  Register-tiled SGEMM (128x64 tile, 8x4 per thread,
// double-buffered shared memory) with fused epilogues:
//   forward  : H = celu(A W + b)
//   head     : e = H3 . w4 + b4 ;  G3 = w4 * celu'(H3)
//   backward : G = (G' W^T) * celu'(H)   (celu' recovered from H itself:
//              1 for H > 0, H/alpha + 1 otherwise)
//   input    : dX (+)= (G1 W1^T) / n_models
#include "mlp_common.cuh"

using namespace fnl;

namespace {

constexpr int BM = 128, BN = 64, BK = 16;
constexpr int TM = 8, TN = 4;  // per-thread tile

enum Epi { EPI_BIAS_CELU = 0, EPI_DCELU = 1, EPI_SCALE_ACC = 2 };

struct GemmArgs {
  const float* A;
  int lda;
  const float* W;      // group-strided weights
  size_t w_group;      // elements between groups
  int ldw;             // row stride of W
  const float* bias;   // group-strided bias (EPI_BIAS_CELU)
  size_t b_group;
  float* C;
  int ldc;
  int K, N;
  const int* tile_species;
  const int* tile_row;
  int group0;          // model * n_species
  float alpha;         // celu alpha or output scale
  float beta;          // EPI_SCALE_ACC: C = beta*C + scale*acc
  float scale;
};

// NT = false: C = A @ W with W [K][N] (row stride ldw)
// NT = true : C = A @ W^T with W [N][K] (row stride ldw)
template <bool NT, int EPI>
__global__ void __launch_bounds__(256) k_sgemm(GemmArgs g) {
  __shared__ float As[2][BK][BM + 4];
  __shared__ float Bs[2][BK][BN + 4];
  const int tile = blockIdx.x;
  const int n0 = blockIdx.y * BN;
  const int row0 = g.tile_row[tile];
  const int grp = g.group0 + g.tile_species[tile];
  const float* W = g.W + (size_t)grp * g.w_group;
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;

  float acc[TM][TN];
#pragma unroll
  for (int a = 0; a < TM; ++a)
#pragma unroll
    for (int b = 0; b < TN; ++b) acc[a][b] = 0.f;

  // global -> register staging
  float ra[8], rb[4];
  auto load_tile = [&](int k0) {
    // A: 128 rows x 16 k ; thread loads 8 elements: rows (tid/16)+16*q, k = tid%16
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      int r = (tid >> 4) + 16 * q, k = k0 + (tid & 15);
      ra[q] = k < g.K ? g.A[(size_t)(row0 + r) * g.lda + k] : 0.f;
    }
    if (!NT) {
      // W[K][N]: 16 k x 64 n; thread loads 4: k = tid/16, n = (tid%16)*4 + q
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int k = k0 + (tid >> 4), n = n0 + (tid & 15) * 4 + q;
        rb[q] = (k < g.K && n < g.N) ? W[(size_t)k * g.ldw + n] : 0.f;
      }
    } else {
      // W[N][K]: 64 n x 16 k ; thread loads 4: n = tid/4 , k = (tid%4)*4 + q
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        int n = n0 + (tid >> 2), k = k0 + (tid & 3) * 4 + q;
        rb[q] = (k < g.K && n < g.N) ? W[(size_t)n * g.ldw + k] : 0.f;
      }
    }
  };
  auto store_tile = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 8; ++q) As[buf][tid & 15][(tid >> 4) + 16 * q] = ra[q];
    if (!NT) {
#pragma unroll
      for (int q = 0; q < 4; ++q) Bs[buf][tid >> 4][(tid & 15) * 4 + q] = rb[q];
    } else {
#pragma unroll
      for (int q = 0; q < 4; ++q) Bs[buf][(tid & 3) * 4 + q][tid >> 2] = rb[q];
    }
  };

  const int nk = (g.K + BK - 1) / BK;
  load_tile(0);
  store_tile(0);
  __syncthreads();
  for (int kt = 0; kt < nk; ++kt) {
    int buf = kt & 1;
    if (kt + 1 < nk) load_tile((kt + 1) * BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float av[TM], bv[TN];
#pragma unroll
      for (int a = 0; a < TM; ++a) av[a] = As[buf][kk][ty * TM + a];
#pragma unroll
      for (int b = 0; b < TN; ++b) bv[b] = Bs[buf][kk][tx * TN + b];
#pragma unroll
      for (int a = 0; a < TM; ++a)
#pragma unroll
        for (int b = 0; b < TN; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
    }
    if (kt + 1 < nk) store_tile(buf ^ 1);
    __syncthreads();
  }

  const float* bias = (EPI == EPI_BIAS_CELU) ? g.bias + (size_t)grp * g.b_group : nullptr;
#pragma unroll
  for (int a = 0; a < TM; ++a) {
    int r = row0 + ty * TM + a;
    float* crow = g.C + (size_t)r * g.ldc;
#pragma unroll
    for (int b = 0; b < TN; ++b) {
      int n = n0 + tx * TN + b;
      if (n >= g.N) continue;
      float v = acc[a][b];
      if (EPI == EPI_BIAS_CELU) {
        crow[n] = celu_f(v + bias[n], g.alpha);
      } else if (EPI == EPI_DCELU) {
        crow[n] = v * dcelu_from_h(crow[n], g.alpha);
      } else {
        crow[n] = (g.beta != 0.f ? g.beta * crow[n] : 0.f) + g.scale * v;
      }
    }
  }
}

// Last layer (width dims[3] -> 1) and its transpose: one warp per row.
__global__ void k_head(float* __restrict__ H3, int ld, int n3, const float* __restrict__ w4,
                       size_t w_group, const float* __restrict__ b4, size_t b_group,
                       const int* __restrict__ tile_species, const int* __restrict__ tile_row,
                       int ntiles, int group0, float alpha, float inv_models, int first_model,
                       float* __restrict__ e_rows) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int tile = warp / 128;
  if (tile >= ntiles) return;
  int r = tile_row[tile] + (warp % 128);
  int grp = group0 + tile_species[tile];
  const float* w = w4 + (size_t)grp * w_group;
  float* h = H3 + (size_t)r * ld;
  float e = 0.f;
  for (int n = lane; n < n3; n += 32) {
    float hv = h[n];
    float wv = w[n];
    e = fmaf(hv, wv, e);
    h[n] = wv * dcelu_from_h(hv, alpha);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if (lane == 0) {
    e += b4[(size_t)grp * b_group];
    e_rows[r] = (first_model ? 0.f : e_rows[r]) + e * inv_models;
  }
}

}  // namespace

size_t fnl_mlp_simt_workspace(int rows, const fennol_mlp_weights* w) {
  return (size_t)rows * (w->dims[1] + w->dims[2] + w->dims[3]) * sizeof(float);
}

int fnl_mlp_simt(int rows, int ntiles, const int* tile_species, const int* tile_row,
                 const fennol_mlp_weights* w, const float* x, float* e_rows, float* dx, void* ws,
                 cudaStream_t st) {
  const int* d = w->dims;
  float* H1 = (float*)ws;
  float* H2 = H1 + (size_t)rows * d[1];
  float* H3 = H2 + (size_t)rows * d[2];
  float* Hs[4] = {nullptr, H1, H2, H3};
  const float alpha = w->celu_alpha;
  const float inv_m = 1.0f / (float)w->n_models;
  for (int m = 0; m < w->n_models; ++m) {
    int g0 = m * w->n_species;
    // forward layers 1..3
    for (int l = 0; l < 3; ++l) {
      GemmArgs a{};
      a.A = l == 0 ? x : Hs[l];
      a.lda = d[l];
      a.W = w->w32[l];
      a.w_group = (size_t)d[l] * d[l + 1];
      a.ldw = d[l + 1];
      a.bias = w->b32[l];
      a.b_group = d[l + 1];
      a.C = Hs[l + 1];
      a.ldc = d[l + 1];
      a.K = d[l];
      a.N = d[l + 1];
      a.tile_species = tile_species;
      a.tile_row = tile_row;
      a.group0 = g0;
      a.alpha = alpha;
      dim3 grid(ntiles, (d[l + 1] + BN - 1) / BN);
      k_sgemm<false, EPI_BIAS_CELU><<<grid, 256, 0, st>>>(a);
      if (cudaGetLastError() != cudaSuccess) return FENNOL_ERR_CUDA;
    }
    // head: energy + G3 (in place of H3)
    {
      int warps = ntiles * 128;
      k_head<<<(warps * 32 + 255) / 256, 256, 0, st>>>(H3, d[3], d[3], w->w32[3], (size_t)d[3], w->b32[3], 1,
                                                       tile_species, tile_row, ntiles, g0, alpha, inv_m,
                                                       m == 0, e_rows);
      if (cudaGetLastError() != cudaSuccess) return FENNOL_ERR_CUDA;
    }
    // backward layers 3..2: G_{l} = (G_{l+1} W_{l+1}^T) * celu'(H_l), in place of H_l
    for (int l = 2; l >= 1; --l) {
      GemmArgs a{};
      a.A = Hs[l + 1];
      a.lda = d[l + 1];
      a.W = w->w32[l];
      a.w_group = (size_t)d[l] * d[l + 1];
      a.ldw = d[l + 1];
      a.C = Hs[l];
      a.ldc = d[l];
      a.K = d[l + 1];
      a.N = d[l];
      a.tile_species = tile_species;
      a.tile_row = tile_row;
      a.group0 = g0;
      a.alpha = alpha;
      dim3 grid(ntiles, (d[l] + BN - 1) / BN);
      k_sgemm<true, EPI_DCELU><<<grid, 256, 0, st>>>(a);
      if (cudaGetLastError() != cudaSuccess) return FENNOL_ERR_CUDA;
    }
    // input gradient dX (+)= G1 W1^T / n_models
    {
      GemmArgs a{};
      a.A = H1;
      a.lda = d[1];
      a.W = w->w32[0];
      a.w_group = (size_t)d[0] * d[1];
      a.ldw = d[1];
      a.C = dx;
      a.ldc = d[0];
      a.K = d[1];
      a.N = d[0];
      a.tile_species = tile_species;
      a.tile_row = tile_row;
      a.group0 = g0;
      a.beta = m == 0 ? 0.f : 1.f;
      a.scale = inv_m;
      dim3 grid(ntiles, (d[0] + BN - 1) / BN);
      k_sgemm<true, EPI_SCALE_ACC><<<grid, 256, 0, st>>>(a);
      if (cudaGetLastError() != cudaSuccess) return FENNOL_ERR_CUDA;
    }
  }
  return FENNOL_OK;
}
