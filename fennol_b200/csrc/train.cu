// Network sweep of the training-loss parameter gradient, on CUDA cores.
//
// FeNNol trains with jax.value_and_grad over a loss that holds forces
// (src/fennol/training/utils.py:140-525, train_step :508): second-order
// differentiation through SpeciesIndexNet (src/fennol/models/misc/nets.py:
// 13-102, 301-426).  With t = dAEV/dx . dL/dF from the AEV tangent kernel,
// the parameter gradient of the loss is the gradient, per species network f,
// of  sum_rows c_e[row] f(a_row) - <grad_a f(a_row), t_row>  (a = AEV row,
// c_e = dL/dE of the row's system).  This file computes it:
//
//   forward    [z_l; zd_l] = [h_{l-1}; hd_{l-1}] W_l (+ b_l on the z rows)
//              h_l = celu(z_l), hd_l = celu'(z_l) zd_l          (l = 1..3)
//   head       seeds hbar_3 = c_e w4, hdbar_3 = -w4; grad w4 = h_3^T c_e - sum hd_3,
//              grad b4 = sum c_e
//   backward   zbar = celu' hbar + celu'' zd hdbar, zdbar = celu' hdbar
//              grad W_l = [h_{l-1}; hd_{l-1}]^T [zbar_l; zdbar_l], grad b_l = sum zbar_l
//              [hbar_{l-1}; hdbar_{l-1}] = [zbar_l; zdbar_l] W_l^T
//
// The activation and its tangent of a species are stacked in one [2R x d]
// buffer, so every product above is one plain GEMM; all species of a batch
// go through one grouped launch per stage (blockIdx.z = species).  GEMMs are
// 128 x 128 shared-memory tiles with 8 x 8 register blocks, float32 or
// float64 arithmetic (the sweep's precision); the weight-gradient products
// (K = all rows of a species) are split along K with the partial products
// summed in a fixed order, so the result is deterministic.
#include <algorithm>

#include "common.cuh"

namespace {

constexpr int kMaxG = 8;   // species per batch
constexpr int BM = 128, BN = 128, BK = 8;
constexpr int kMaxSplit = 8;   // K slices of one GEMM (partials summed in order)

template <typename T>
struct GemmGroups {
  const T* a[kMaxG];
  const T* b[kMaxG];
  T* c[kMaxG];
  const T* bias[kMaxG];
  T* part[kMaxG];   // [splits][m][n] partial products when splits > 1
  int m[kMaxG], k[kMaxG], lda[kMaxG], ldb[kMaxG], ldc[kMaxG], bias_rows[kMaxG];
  int splits;
};

template <typename T>
__device__ __forceinline__ void lds4(const T* p, T* v) {
  if constexpr (sizeof(T) == 4) {
    const float4 q = *reinterpret_cast<const float4*>(p);
    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
  } else {
    const double2 q0 = *reinterpret_cast<const double2*>(p);
    const double2 q1 = *reinterpret_cast<const double2*>(p + 2);
    v[0] = q0.x, v[1] = q0.y, v[2] = q1.x, v[3] = q1.y;
  }
}

// C[m][n] = sum_k op(A)[m][k] op(B)[k][n] (+ bias[n] for m < bias_rows);
// op(A) = A[k][m] when TA (A stored k-major), A[m][k] otherwise; op(B) =
// B[n][k] when TB, B[k][n] otherwise.  128 x 128 tiles, 256 threads with an
// 8 x 8 register block each (rows ty*4 and 64 + ty*4, columns tx*4 and
// 64 + tx*4), the next K-slice prefetched into registers while the current
// one is multiplied.  blockIdx.z = group * splits + split; with splits > 1
// each split writes its partial product and k_split_sum adds them in order.
template <typename T, bool TA, bool TB>
__global__ void __launch_bounds__(256) k_gemm(const GemmGroups<T> g, int N) {
  const int grp = blockIdx.z / g.splits, split = blockIdx.z % g.splits;
  const int M = g.m[grp], K = g.k[grp];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  if (m0 >= M) return;
  const int kper = ((K + g.splits - 1) / g.splits + BK - 1) / BK * BK;
  const int kb = split * kper, ke = min(K, kb + kper);
  const T* __restrict__ A = g.a[grp];
  const T* __restrict__ B = g.b[grp];
  const int lda = g.lda[grp], ldb = g.ldb[grp];
  __shared__ __align__(16) T As[2][BK][BM];
  __shared__ __align__(16) T Bs[2][BK][BN];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // element e = tid + 256 i (i < 4) of a BK x 128 slice
  auto fetch = [&](int k0, T* ra, T* rb) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int e = tid + 256 * i;
      int mm, kk;
      if (TA) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
      const int m = m0 + mm, k = k0 + kk;
      ra[i] = (m < M && k < ke) ? (TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]) : T(0);
      int nn;
      if (TB) { kk = e % BK; nn = e / BK; } else { nn = e % BN; kk = e / BN; }
      const int n = n0 + nn, k2 = k0 + kk;
      rb[i] = (n < N && k2 < ke) ? (TB ? B[(size_t)n * ldb + k2] : B[(size_t)k2 * ldb + n]) : T(0);
    }
  };
  auto store = [&](int buf, const T* ra, const T* rb) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int e = tid + 256 * i;
      if (TA) As[buf][e / BM][e % BM] = ra[i]; else As[buf][e % BK][e / BK] = ra[i];
      if (TB) Bs[buf][e % BK][e / BK] = rb[i]; else Bs[buf][e / BN][e % BN] = rb[i];
    }
  };
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = T(0);
  T ra[4], rb[4];
  int buf = 0;
  if (kb < ke) {
    fetch(kb, ra, rb);
    store(0, ra, rb);
  }
  __syncthreads();
  for (int k0 = kb; k0 < ke; k0 += BK) {
    const bool more = k0 + BK < ke;
    if (more) fetch(k0 + BK, ra, rb);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[8], b[8];
      lds4(&As[buf][kk][ty * 4], a);
      lds4(&As[buf][kk][64 + ty * 4], a + 4);
      lds4(&Bs[buf][kk][tx * 4], b);
      lds4(&Bs[buf][kk][64 + tx * 4], b + 4);
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] += a[i] * b[j];
    }
    if (more) store(buf ^ 1, ra, rb);
    __syncthreads();
    buf ^= 1;
  }
  const bool partial = g.splits > 1;
  T* __restrict__ C = partial ? g.part[grp] + (size_t)split * M * N : g.c[grp];
  const int ldc = partial ? N : g.ldc[grp];
  const T* bias = partial ? nullptr : g.bias[grp];
  const int brows = g.bias_rows[grp];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int m = m0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + i - 4);
    if (m >= M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = n0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + j - 4);
      if (n >= N) continue;
      T v = acc[i][j];
      if (bias && m < brows) v += bias[n];
      C[(size_t)m * ldc + n] = v;
    }
  }
}

// C = sum over splits of the partial products, in split order (+ bias)
template <typename T>
__global__ void k_split_sum(const GemmGroups<T> g, int N) {
  const int grp = blockIdx.y;
  const int M = g.m[grp];
  const size_t total = (size_t)M * N;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const int m = (int)(i / N), n = (int)(i % N);
    T v = T(0);
    for (int s = 0; s < g.splits; ++s) v += g.part[grp][(size_t)s * total + i];
    if (g.bias[grp] && m < g.bias_rows[grp]) v += g.bias[grp][n];
    g.c[grp][(size_t)m * g.ldc[grp] + n] = v;
  }
}

template <typename T>
struct Elem {
  const T* in0[kMaxG];
  const T* in1[kMaxG];
  T* out0[kMaxG];
  T* out1[kMaxG];
  int rows[kMaxG];
  int row0[kMaxG];
};

// [x_rows; t_rows] of each species (columns [0, F)) into one [2R x F] buffer
template <typename T>
__global__ void k_stack(const Elem<T> e, int F, int ld) {
  const int grp = blockIdx.y, R = e.rows[grp];
  const size_t total = (size_t)R * F;
  const T* x = e.in0[grp] + (size_t)e.row0[grp] * ld;
  const T* t = e.in1[grp] + (size_t)e.row0[grp] * ld;
  T* out = e.out0[grp];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / F, f = i % F;
    out[i] = x[r * ld + f];
    out[total + i] = t[r * ld + f];
  }
}

template <typename T>
__device__ __forceinline__ void celu3(T z, T alpha, T& h, T& d1, T& d2) {
  const T e = exp((z < T(0) ? z : T(0)) / alpha);
  h = z > T(0) ? z : alpha * (e - T(1));
  d1 = z > T(0) ? T(1) : e;
  d2 = z > T(0) ? T(0) : e / alpha;
}

// [z; zd] (2R x d) -> [celu(z); celu'(z) zd]
template <typename T>
__global__ void k_celu_fwd(const Elem<T> e, int d, T alpha) {
  const int grp = blockIdx.y;
  const size_t total = (size_t)e.rows[grp] * d;
  const T* zc = e.in0[grp];
  T* hc = e.out0[grp];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    T h, d1, d2;
    celu3(zc[i], alpha, h, d1, d2);
    hc[i] = h;
    hc[total + i] = d1 * zc[total + i];
  }
}

// [zbar; zdbar] from [hbar; hdbar] and [z; zd]
template <typename T>
__global__ void k_celu_bwd(const Elem<T> e, int d, T alpha) {
  const int grp = blockIdx.y;
  const size_t total = (size_t)e.rows[grp] * d;
  const T* hb = e.in0[grp];
  const T* zc = e.in1[grp];
  T* zb = e.out0[grp];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    T h, d1, d2;
    celu3(zc[i], alpha, h, d1, d2);
    const T hdbar = hb[total + i];
    zb[i] = d1 * hb[i] + d2 * zc[total + i] * hdbar;
    zb[total + i] = d1 * hdbar;
  }
}

// head seeds: hbar = c_e w4, hdbar = -w4 through the last hidden CELU, and
// the vector [c_e; -1] whose product with [h; hd]^T is the w4 gradient
template <typename T>
__global__ void k_head_seed(const Elem<T> e, int d, T alpha, const T* c_row) {
  const int grp = blockIdx.y, R = e.rows[grp];
  const size_t total = (size_t)R * d;
  const T* zc = e.in0[grp];
  T* zb = e.out0[grp];
  T* v = e.out1[grp];
  const T* w = e.in1[grp];   // the last layer's kernel (d x 1)
  const T* ce = c_row + e.row0[grp];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / d, j = i % d;
    T h, d1, d2;
    celu3(zc[i], alpha, h, d1, d2);
    const T hbar = ce[r] * w[j], hdbar = -w[j];
    zb[i] = d1 * hbar + d2 * zc[total + i] * hdbar;
    zb[total + i] = d1 * hdbar;
    if (j == 0) {
      v[r] = ce[r];
      v[R + r] = T(-1);
    }
  }
}

// out[j] = sum over the first R rows of in[r][j] (d columns), fixed order
template <typename T>
__global__ void __launch_bounds__(256) k_colsum(const Elem<T> e, int d) {
  const int grp = blockIdx.y, R = e.rows[grp];
  const T* in = e.in0[grp];
  T* out = e.out0[grp];
  const int j = blockIdx.x * 32 + (threadIdx.x & 31);
  const int slice = threadIdx.x >> 5;
  __shared__ T part[8][32];
  T s = T(0);
  if (j < d)
    for (int r = slice; r < R; r += 8) s += in[(size_t)r * d + j];
  part[slice][threadIdx.x & 31] = s;
  __syncthreads();
  if (slice == 0 && j < d) {
    T t = T(0);
#pragma unroll
    for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x & 31];
    out[j] = t;
  }
}

inline dim3 egrid(size_t total, int groups) {
  size_t b = (total + 255) / 256;
  if (b > 148 * 8) b = 148 * 8;
  if (b < 1) b = 1;
  return dim3((unsigned)b, (unsigned)groups);
}

// One grouped GEMM launch; with splits > 1 the caller has set g.part and the
// partial products are summed in split order by a second launch.
template <typename T, bool TA, bool TB>
int gemm(GemmGroups<T> g, int ng, int N, int Mmax, int splits, cudaStream_t st) {
  if (ng == 0 || N <= 0 || Mmax <= 0) return FENNOL_OK;
  g.splits = splits;
  dim3 grid((N + BN - 1) / BN, (Mmax + BM - 1) / BM, ng * splits);
  k_gemm<T, TA, TB><<<grid, 256, 0, st>>>(g, N);
  if (splits > 1) k_split_sum<T><<<egrid((size_t)Mmax * N, ng), 256, 0, st>>>(g, N);
  return cudaGetLastError() == cudaSuccess ? FENNOL_OK : FENNOL_ERR_CUDA;
}

// K slices of the weight-gradient products (K = 2R rows): enough blocks to
// fill the SMs, at least 512 rows per slice
inline int splits_for(int kmax) {
  int s = (kmax + 511) / 512;
  return s < 1 ? 1 : (s > kMaxSplit ? kMaxSplit : s);
}

// workspace carve-up of one species with R rows (elements of T)
struct Carve {
  size_t h0, z[4], h[4], zb[4], hb[4], v, part, total;
};

Carve carve(const int* dims, int R) {
  Carve c{};
  size_t o = 0;
  auto take = [&](size_t n) {
    size_t p = o;
    o += (n + 31) / 32 * 32;  // 256-byte alignment for doubles
    return p;
  };
  const size_t R2 = 2 * (size_t)R;
  c.h0 = take(R2 * dims[0]);
  for (int l = 1; l <= 3; ++l) {
    c.z[l] = take(R2 * dims[l]);
    c.h[l] = take(R2 * dims[l]);
    c.zb[l] = take(R2 * dims[l]);
  }
  for (int l = 1; l <= 2; ++l) c.hb[l] = take(R2 * dims[l]);
  c.v = take(R2);
  size_t mn = 0;
  for (int l = 1; l <= 4; ++l) mn = std::max(mn, (size_t)dims[l - 1] * dims[l]);
  c.part = take((size_t)kMaxSplit * mn);
  c.total = o;
  return c;
}

template <typename T>
int run(const fennol_net_train* net, const int* host_row0, const int* host_rows, const void* x_, const void* t_,
        int ld, const void* c_row_, void* ws, cudaStream_t st) {
  const int* d = net->dims;
  const T alpha = (T)net->celu_alpha;
  const T* x = (const T*)x_;
  const T* t = (const T*)t_;
  const T* c_row = (const T*)c_row_;
  // the species with rows, in order
  int sp[kMaxG], ng = 0, Rmax = 0;
  Carve cv[kMaxG];
  T* base[kMaxG];
  size_t off = 0;
  for (int s = 0; s < net->n_species; ++s) {
    if (host_rows[s] <= 0) continue;
    sp[ng] = s;
    cv[ng] = carve(d, host_rows[s]);
    base[ng] = (T*)ws + off;
    off += cv[ng].total;
    Rmax = host_rows[s] > Rmax ? host_rows[s] : Rmax;
    ++ng;
  }
  if (ng == 0) return FENNOL_OK;
  auto W = [&](int l, int gi) { return (const T*)net->w[l][sp[gi]]; };
  auto Bv = [&](int l, int gi) { return (const T*)net->b[l][sp[gi]]; };
  int rc;
  // stack [x; t]
  {
    Elem<T> e{};
    for (int gi = 0; gi < ng; ++gi) {
      e.in0[gi] = x;
      e.in1[gi] = t;
      e.out0[gi] = base[gi] + cv[gi].h0;
      e.rows[gi] = host_rows[sp[gi]];
      e.row0[gi] = host_row0[sp[gi]];
    }
    k_stack<T><<<egrid((size_t)Rmax * d[0], ng), 256, 0, st>>>(e, d[0], ld);
  }
  // forward through the three hidden layers
  for (int l = 1; l <= 3; ++l) {
    GemmGroups<T> g{};
    for (int gi = 0; gi < ng; ++gi) {
      const int R = host_rows[sp[gi]];
      g.a[gi] = base[gi] + (l == 1 ? cv[gi].h0 : cv[gi].h[l - 1]);
      g.b[gi] = W(l - 1, gi);
      g.c[gi] = base[gi] + cv[gi].z[l];
      g.bias[gi] = Bv(l - 1, gi);
      g.m[gi] = 2 * R;
      g.k[gi] = d[l - 1];
      g.lda[gi] = d[l - 1];
      g.ldb[gi] = d[l];
      g.ldc[gi] = d[l];
      g.bias_rows[gi] = R;
    }
    if ((rc = gemm<T, false, false>(g, ng, d[l], 2 * Rmax, 1, st))) return rc;
    Elem<T> e{};
    for (int gi = 0; gi < ng; ++gi) {
      e.in0[gi] = base[gi] + cv[gi].z[l];
      e.out0[gi] = base[gi] + cv[gi].h[l];
      e.rows[gi] = host_rows[sp[gi]];
    }
    k_celu_fwd<T><<<egrid((size_t)Rmax * d[l], ng), 256, 0, st>>>(e, d[l], alpha);
  }
  // head: seeds into the last hidden layer, w4 and b4 gradients
  {
    Elem<T> e{};
    for (int gi = 0; gi < ng; ++gi) {
      e.in0[gi] = base[gi] + cv[gi].z[3];
      e.in1[gi] = W(3, gi);
      e.out0[gi] = base[gi] + cv[gi].zb[3];
      e.out1[gi] = base[gi] + cv[gi].v;
      e.rows[gi] = host_rows[sp[gi]];
      e.row0[gi] = host_row0[sp[gi]];
    }
    k_head_seed<T><<<egrid((size_t)Rmax * d[3], ng), 256, 0, st>>>(e, d[3], alpha, c_row);
    // grad w4 = [h3; hd3]^T [c_e; -1]
    GemmGroups<T> g{};
    for (int gi = 0; gi < ng; ++gi) {
      const int R = host_rows[sp[gi]];
      g.a[gi] = base[gi] + cv[gi].h[3];
      g.b[gi] = base[gi] + cv[gi].v;
      g.c[gi] = (T*)net->gw[3][sp[gi]];
      g.part[gi] = base[gi] + cv[gi].part;
      g.m[gi] = d[3];
      g.k[gi] = 2 * R;
      g.lda[gi] = d[3];
      g.ldb[gi] = 1;
      g.ldc[gi] = 1;
    }
    if ((rc = gemm<T, true, false>(g, ng, 1, d[3], splits_for(2 * Rmax), st))) return rc;
    // grad b4 = sum of c_e over the species' rows
    Elem<T> c{};
    for (int gi = 0; gi < ng; ++gi) {
      c.in0[gi] = c_row + host_row0[sp[gi]];
      c.out0[gi] = (T*)net->gb[3][sp[gi]];
      c.rows[gi] = host_rows[sp[gi]];
    }
    k_colsum<T><<<dim3(1, ng), 256, 0, st>>>(c, 1);
  }
  // backward through the hidden layers
  for (int l = 3; l >= 1; --l) {
    // grad W_{l-1} = [h; hd]_{l-1}^T [zbar; zdbar]_l, straight into the output
    GemmGroups<T> g{};
    for (int gi = 0; gi < ng; ++gi) {
      const int R = host_rows[sp[gi]];
      g.a[gi] = base[gi] + (l == 1 ? cv[gi].h0 : cv[gi].h[l - 1]);
      g.b[gi] = base[gi] + cv[gi].zb[l];
      g.c[gi] = (T*)net->gw[l - 1][sp[gi]];
      g.part[gi] = base[gi] + cv[gi].part;
      g.m[gi] = d[l - 1];
      g.k[gi] = 2 * R;
      g.lda[gi] = d[l - 1];
      g.ldb[gi] = d[l];
      g.ldc[gi] = d[l];
    }
    if ((rc = gemm<T, true, false>(g, ng, d[l], d[l - 1], splits_for(2 * Rmax), st))) return rc;
    Elem<T> c{};
    for (int gi = 0; gi < ng; ++gi) {
      c.in0[gi] = base[gi] + cv[gi].zb[l];
      c.out0[gi] = (T*)net->gb[l - 1][sp[gi]];
      c.rows[gi] = host_rows[sp[gi]];
    }
    k_colsum<T><<<dim3((d[l] + 31) / 32, ng), 256, 0, st>>>(c, d[l]);
    if (l == 1) break;
    // [hbar; hdbar]_{l-1} = [zbar; zdbar]_l W_{l-1}^T, then through CELU
    GemmGroups<T> h{};
    for (int gi = 0; gi < ng; ++gi) {
      const int R = host_rows[sp[gi]];
      h.a[gi] = base[gi] + cv[gi].zb[l];
      h.b[gi] = W(l - 1, gi);
      h.c[gi] = base[gi] + cv[gi].hb[l - 1];
      h.m[gi] = 2 * R;
      h.k[gi] = d[l];
      h.lda[gi] = d[l];
      h.ldb[gi] = d[l];
      h.ldc[gi] = d[l - 1];
    }
    if ((rc = gemm<T, false, true>(h, ng, d[l - 1], 2 * Rmax, 1, st))) return rc;
    Elem<T> e{};
    for (int gi = 0; gi < ng; ++gi) {
      e.in0[gi] = base[gi] + cv[gi].hb[l - 1];
      e.in1[gi] = base[gi] + cv[gi].z[l - 1];
      e.out0[gi] = base[gi] + cv[gi].zb[l - 1];
      e.rows[gi] = host_rows[sp[gi]];
    }
    k_celu_bwd<T><<<egrid((size_t)Rmax * d[l - 1], ng), 256, 0, st>>>(e, d[l - 1], alpha);
  }
  return cudaGetLastError() == cudaSuccess ? FENNOL_OK : FENNOL_ERR_CUDA;
}

bool net_ok(const fennol_net_train* net) {
  if (!net || net->n_species < 1 || net->n_species > kMaxG || net->dims[4] != 1) return false;
  for (int l = 0; l < 4; ++l)
    if (net->dims[l] <= 0) return false;
  return true;
}

size_t elem_size(const fennol_net_train* net) { return net->is_double ? sizeof(double) : sizeof(float); }

}  // namespace

extern "C" size_t fennol_net_loss_grad_workspace_bytes(const fennol_net_train* net, const int* host_rows) {
  if (!net_ok(net) || !host_rows) return 0;
  size_t n = 0;
  for (int s = 0; s < net->n_species; ++s)
    if (host_rows[s] > 0) n += carve(net->dims, host_rows[s]).total;
  return n * elem_size(net) + 256;
}

extern "C" int fennol_net_loss_grad(const fennol_net_train* net, const int* host_row0, const int* host_rows,
                                    const void* x, const void* t, int ld, const void* c_row, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  if (!net_ok(net) || !host_row0 || !host_rows) return FENNOL_ERR_INVALID;
  if (ld < net->dims[0]) return FENNOL_ERR_INVALID;
  bool any = false;
  for (int s = 0; s < net->n_species; ++s) {
    if (host_rows[s] < 0 || host_row0[s] < 0) return FENNOL_ERR_INVALID;
    if (host_rows[s] == 0) continue;
    any = true;
    for (int l = 0; l < 4; ++l)
      if (!net->w[l][s] || !net->b[l][s] || !net->gw[l][s] || !net->gb[l][s]) return FENNOL_ERR_INVALID;
  }
  if (!any) return FENNOL_OK;
  if (!x || !t || !c_row || !workspace) return FENNOL_ERR_INVALID;
  if (((uintptr_t)workspace & 255) != 0) return FENNOL_ERR_INVALID;
  if (workspace_bytes < fennol_net_loss_grad_workspace_bytes(net, host_rows)) return FENNOL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  return net->is_double ? run<double>(net, host_row0, host_rows, x, t, ld, c_row, workspace, st)
                        : run<float>(net, host_row0, host_rows, x, t, ld, c_row, workspace, st);
}
