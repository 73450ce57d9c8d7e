// ANI atomic environment vectors on sm_100a: forward and adjoint (forces).
//
// Replaces ANIAEV.__call__ (src/fennol/models/embeddings/ani.py:47-142), the
// graph processors it reads (GraphProcessor preprocessing.py:719-777,
// GraphFilterProcessor :979-1043, GraphAngularExtension :1085-1276,
// GraphAngleProcessor :1294-1317), the cosine SwitchFunction
// (misc/misc.py:617-716) and, in the backward kernel, the reverse-mode
// transpose jax.grad takes through all of them (fennix.py:260-272).
//
// Layout: one warp per centre atom.  The warp streams the atom's radial row,
// forms the angular sub-list (d^2 < rca^2, same float32 arithmetic as the
// reference filter) in shared memory, enumerates all unordered neighbour
// pairs (the triplets) on chip, and accumulates the 1008 features in shared
// memory with one feature column per lane, so the forward needs no atomics.
// cos(theta - Z) is expanded as cos(theta)cos(Z) + sin(theta)sin(Z) with
// cos(theta) = 0.95 * cos_angle, which removes arccos/cos from the inner loop.
#include <cmath>

#include "common.cuh"

using namespace fnl;

namespace {

constexpr int kAevWarps = 8;
constexpr int kMaxS = 8;
constexpr int kMaxP = kMaxS * (kMaxS + 1) / 2;
// Angular neighbours a centre's staging holds: the row capacity, at most
// FENNOL_MAX_ANGULAR_NEIGHBORS.  A centre has no more angular neighbours than
// radial ones, so rows of up to that capacity cannot overflow it.
constexpr int kCapAMax = FENNOL_MAX_ANGULAR_NEIGHBORS;
__host__ __device__ __forceinline__ int ang_cap(int cap) { return cap < kCapAMax ? cap : kCapAMax; }

struct AevConst {
  int S, P, RD, AD, AS, F;
  float rc, rca, rc2, rca2;   // cutoffs and float32 thresholds
  float pi_rc, pi_rca;        // pi / cutoff
  float eta_r, eta_a, zeta, c_ang;  // c_ang = 2^(1-zeta)
  int zeta_n;                       // floor(zeta) and zeta - floor(zeta)
  float zeta_f;
  int zeta1_n;                      // the same split of zeta - 1
  float zeta1_f;
  float dra, gc2a;                  // angular shift spacing, exp(-2 eta_a dra^2)
  float drr, gc2r, inv_drr, lim_r;  // radial: spacing, exp(-2 eta_r drr^2), 1 / drr, sqrt(80 / eta_r)
  float shift_r[32];
  float shift_a[32];
  float cosz[32], sinz[32];
};

bool make_const(const fennol_aev_params* p, AevConst* k) {
  if (!p) return false;
  int S = p->num_species, RD = p->radial_divisions, AD = p->angular_divisions, AS = p->angle_sections;
  if (S < 1 || S > kMaxS) return false;
  if (!(RD == 16 || RD == 32)) return false;
  if (AD * AS != 32 || AD < 1 || AS < 1) return false;
  if (!(p->radial_cutoff > 0) || !(p->angular_cutoff > 0) || p->angular_cutoff > p->radial_cutoff)
    return false;
  k->S = S;
  k->P = S * (S + 1) / 2;
  k->RD = RD;
  k->AD = AD;
  k->AS = AS;
  k->F = S * RD + k->P * AD * AS;
  k->rc = (float)p->radial_cutoff;
  k->rca = (float)p->angular_cutoff;
  k->rc2 = (float)(p->radial_cutoff * p->radial_cutoff);
  k->rca2 = (float)(p->angular_cutoff * p->angular_cutoff);
  k->pi_rc = (float)(M_PI / p->radial_cutoff);
  k->pi_rca = (float)(M_PI / p->angular_cutoff);
  k->eta_r = p->radial_eta;
  k->eta_a = p->angular_eta;
  k->zeta = p->zeta;
  k->c_ang = (float)std::pow(2.0, 1.0 - (double)p->zeta);
  {
    double zn = std::floor((double)p->zeta);
    k->zeta_n = (int)zn;
    k->zeta_f = (float)((double)p->zeta - zn);
    double z1 = std::floor((double)p->zeta - 1.0);
    k->zeta1_n = (int)z1;
    k->zeta1_f = (float)((double)p->zeta - 1.0 - z1);
    if (p->zeta < 1.0f || p->zeta > 64.0f) return false;
  }
  {
    const double dra = (p->angular_cutoff - p->angular_start) / AD;
    k->dra = (float)dra;
    k->gc2a = (float)std::exp(-2.0 * (double)p->angular_eta * dra * dra);
    const double drr = (p->radial_cutoff - p->radial_start) / RD;
    k->drr = (float)drr;
    k->gc2r = (float)std::exp(-2.0 * (double)p->radial_eta * drr * drr);
    k->inv_drr = (float)(1.0 / drr);
    k->lim_r = (float)std::sqrt(80.0 / (double)p->radial_eta);
  }
  for (int r = 0; r < 32; ++r) {
    k->shift_r[r] = r < RD ? (float)(p->radial_start + (p->radial_cutoff - p->radial_start) * r / RD) : 0.f;
    k->shift_a[r] = r < AD ? (float)(p->angular_start + (p->angular_cutoff - p->angular_start) * r / AD) : 0.f;
    double z = M_PI * r / AS + M_PI / (2.0 * AS);
    k->cosz[r] = r < AS ? (float)std::cos(z) : 0.f;
    k->sinz[r] = r < AS ? (float)std::sin(z) : 0.f;
  }
  return true;
}

__device__ __forceinline__ void load_cell(const float* sys_cell, int b, float* c) {
  if (sys_cell) {
#pragma unroll
    for (int k = 0; k < 9; ++k) c[k] = __ldg(sys_cell + 9 * b + k);
  } else {
#pragma unroll
    for (int k = 0; k < 9; ++k) c[k] = 0.f;
  }
}

// Edge vector x_j - x_i + s @ cell with the reference filter's float32 arithmetic.
__device__ __forceinline__ void edge_vec(float4 pi, float4 pj, unsigned sh, const float* c, float& vx,
                                         float& vy, float& vz) {
  vx = __fsub_rn(pj.x, pi.x);
  vy = __fsub_rn(pj.y, pi.y);
  vz = __fsub_rn(pj.z, pi.z);
  if (sh) {
    int sx, sy, sz;
    unpack_shift(sh, sx, sy, sz);
    add_shift(vx, vy, vz, (float)sx, (float)sy, (float)sz, c);
  }
}

__device__ __forceinline__ __nv_bfloat16 to_bf16(float x) { return __float2bfloat16_rn(x); }

// ------------------------------------------------------------------------------
// Species-sorted staging shared by the forward and adjoint kernels.
//
// The warp streams the atom's radial row once, computes the edge geometry with
// the reference's float32 arithmetic and writes it unsorted to `tmp`; a
// ballot-based counting sort then places the radial neighbours (d, 0.25 fc)
// and the angular ones (unit vector, d, fc, slot) grouped by species, so
// every species block and every species-pair block of triplets is contiguous.
// ------------------------------------------------------------------------------
struct Stage {
  float4* tmp;   // [cap] (vx, vy, vz, d2) unsorted
  int* tkey;     // [cap] species | angular<<8
  float2* rd;    // [cap] radial (d, 0.25*fc) sorted by species
  float4* au;    // [capa] angular (ux, uy, uz, d) sorted by species
  float2* af;    // [capa] angular (fc, dfc)
  int* aslot;    // [capa] radial row position of each angular neighbour
  int* cntw;     // [32] per-species counters
  int* rslot;    // [cap] radial row position of each sorted radial entry (tangent kernel only)
  int capa;      // angular capacity, ang_cap(cap)
};

// `with_rd`: the sorted radial entries (d, 0.25 fc) are kept (forward and
// tangent); the adjoint works from the unsorted rows and leaves them out.
__host__ __device__ __forceinline__ size_t stage_bytes(int cap, bool with_rd = true) {
  // rounded to 16 bytes so that every per-warp carve-up keeps float4 alignment
  return ((size_t)cap * (16 + 4 + (with_rd ? 8 : 0)) + (size_t)ang_cap(cap) * (16 + 8 + 4) + 32 * 4 + 15) / 16 * 16;
}

__device__ __forceinline__ Stage carve_stage(char* base, int cap, bool with_rd = true) {
  Stage st;
  st.tmp = (float4*)base;
  st.au = (float4*)(base + (size_t)cap * 16);
  const int capa = ang_cap(cap);
  char* next = base + (size_t)cap * 16 + (size_t)capa * 16;
  st.rd = with_rd ? (float2*)next : nullptr;
  if (with_rd) next += (size_t)cap * 8;
  st.af = (float2*)next;
  st.tkey = (int*)((char*)st.af + (size_t)capa * 8);
  st.aslot = st.tkey + cap;
  st.cntw = st.aslot + capa;
  st.rslot = nullptr;
  st.capa = capa;
  return st;
}

// Gaussian terms use the accurate expf: their arguments reach -50 and the
// SFU-only __expf loses ~|x|*2^-24 of relative accuracy there.
__device__ __forceinline__ float fexp(float x) { return expf(x); }
__device__ __forceinline__ float exp2f_approx_pos(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Gaussians B[r] = exp(-eta (x0 - r dr)^2) of uniformly spaced shifts from
// two exponentials: B[r+1] = B[r] g[r] with g[r] = exp(eta dr (2 (x0 - r dr) - dr))
// and g[r+1] = g[r] c2, c2 = exp(-2 eta dr^2).  Every B[r] and g[r] stays below
// its start value, so nothing overflows; when B[0] would be tiny (its
// exponent below -80) the terms are evaluated one by one instead.
template <int N>
__device__ __forceinline__ void gauss_chain(float x0, float eta, float dr, float c2, float* B) {
  if (eta * x0 * x0 > 80.f) {
#pragma unroll
    for (int r = 0; r < N; ++r) {
      const float x = x0 - (float)r * dr;
      B[r] = fexp(-eta * x * x);
    }
    return;
  }
  float b = fexp(-eta * x0 * x0);
  float g = fexp(eta * dr * (2.f * x0 - dr));
#pragma unroll
  for (int r = 0; r < N; ++r) {
    B[r] = b;
    b *= g;
    g *= c2;
  }
}

// The same for shifts spread over a wider range (the radial ones), where the
// first term underflows for most distances: B[r] = exp(-eta (x0 - r dr)^2),
// r < N, from two exponentials.  Terms below exp(-80) (< 2e-35, far below anything a
// float32 sum of the others registers) are 0; from the first shift r0 at or
// above that bound the chain B[r+1] = B[r] g[r], g[r] = exp(eta dr (2 (x0 -
// r dr) - dr)), g[r+1] = g[r] c2 with c2 = exp(-2 eta dr^2) takes over.  B
// rises to at most 1 and then falls, and g stays below exp(2 eta dr (lim +
// dr)), so nothing overflows.  lim = sqrt(80 / eta), inv_dr = 1 / dr.
template <int N>
__device__ __forceinline__ void gauss_chain_from(float x0, float eta, float dr, float inv_dr, float c2, float lim,
                                                 float* B) {
  const float rs = ceilf((x0 - lim) * inv_dr);
  const int r0 = rs <= 0.f ? 0 : (rs >= (float)N ? N : (int)rs);
  const float xs = x0 - (float)r0 * dr;
  float b = fexp(-eta * xs * xs);
  float g = fexp(eta * dr * (2.f * xs - dr));
#pragma unroll
  for (int r = 0; r < N; ++r) {
    const bool on = r >= r0;
    B[r] = on ? b : 0.f;
    if (on) {
      b *= g;
      g *= c2;
    }
  }
}

// x^zeta for x >= 0 as x^n * x^f with n = floor(zeta): the integer power by
// repeated squaring (a few roundings) and only the fractional power through
// the SFU exp2/log2 approximations, whose log2 error is then scaled by f < 1
// instead of by zeta (14.1).  N >= 0 is n known at compile time (the kernels
// built for the ANI-2x exponent): the same products in the same order, with
// the bit tests and unused squarings gone; N < 0 reads n at run time.
template <int N>
__device__ __forceinline__ float zeta_pow(float x, int n, float f) {
  if (x <= 0.f) return 0.f;
  float r = 1.f, b = x;
#pragma unroll
  for (int k = 0; k < 6; ++k) {  // n < 64
    const bool bit = N >= 0 ? ((N >> k) & 1) != 0 : ((n >> k) & 1) != 0;
    r = bit ? r * b : r;
    if (N >= 0 && (N >> (k + 1)) == 0) break;
    b *= b;
  }
  return f != 0.f ? r * exp2f_approx_pos(f * __log2f(x)) : r;
}

// integer part of zeta - 1 for a compile-time integer part ZN of zeta
__host__ __device__ constexpr int zn_minus1(int zn) { return zn >= 0 ? zn - 1 : -1; }

// Warp-collective: stage row i.  Returns, in lanes s < S, the per-species
// radial and angular counts and exclusive offsets.  Lanes holding the same
// species are grouped with __match_any_sync; per-warp counters live in `cntw`.
template <bool kGrad, bool kRslot = false, bool kRd = true>
__device__ __forceinline__ void stage_row(const Stage& st, int* cntw, const float4* __restrict__ xyzs, float4 pi,
                                          const float* c, const int* __restrict__ nbr_j,
                                          const unsigned* __restrict__ nbr_shift, size_t row, int cnt,
                                          const AevConst& K, int lane, int& cnt_r, int& off_r, int& cnt_a,
                                          int& off_a, int& na_total) {
  const int S = K.S;
  // cntw[0..S): radial counts, [S..2S): angular counts, [2S..4S): running offsets
  if (lane < 4 * S) cntw[lane] = 0;
  // gather: the edge geometry of every row entry.  No warp-collective step
  // here, so the loads of consecutive rounds are in flight together.
#pragma unroll 2
  for (int k = lane; k < cnt; k += 32) {
    const int j = __ldg(nbr_j + row + k);
    const unsigned sh = __ldg(nbr_shift + row + k);
    const float4 pj = xyzs[j];
    float vx, vy, vz;
    edge_vec(pi, pj, sh, c, vx, vy, vz);
    const float d2 = dist2_exact(vx, vy, vz);
    st.tmp[k] = make_float4(vx, vy, vz, d2);
    st.tkey[k] = __float_as_int(pj.w) | ((d2 < K.rca2) << 8);
  }
  __syncwarp();
  const unsigned lt = (1u << lane) - 1u;
  // count the entries per species (radial) and per species within rca (angular)
  for (int k0 = 0; k0 < cnt; k0 += 32) {
    const int k = k0 + lane;
    const int key = k < cnt ? st.tkey[k] : -1;
    const unsigned grp = __match_any_sync(0xffffffffu, key);
    if (key >= 0 && (grp & lt) == 0) {  // group leader (two groups may share a species)
      const int sj = key & 0xFF;
      if (key >> 8) atomicAdd(cntw + S + sj, __popc(grp));
      atomicAdd(cntw + sj, __popc(grp));
    }
    __syncwarp();
  }
  // the angular key groups also counted towards radial above; radial counts are
  // per species regardless of the angular bit
  int cr = lane < S ? cntw[lane] : 0;
  int ca = lane < S ? cntw[S + lane] : 0;
  int ir = cr, ia = ca;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t1 = __shfl_up_sync(0xffffffffu, ir, o);
    int t2 = __shfl_up_sync(0xffffffffu, ia, o);
    if (lane >= o) {
      ir += t1;
      ia += t2;
    }
  }
  cnt_r = cr;
  cnt_a = ca;
  off_r = ir - cr;
  off_a = ia - ca;
  na_total = __shfl_sync(0xffffffffu, ia, S - 1);
  if (lane < S) {
    cntw[2 * S + lane] = off_r;
    cntw[3 * S + lane] = off_a;
  }
  __syncwarp();
  for (int k0 = 0; k0 < cnt; k0 += 32) {
    const int k = k0 + lane;
    const int key = k < cnt ? st.tkey[k] : -1;
    const int sj = key & 0xFF;
    const int isang = key >= 0 ? (key >> 8) : 0;
    // radial position: group by species only
    const unsigned gr_ = __match_any_sync(0xffffffffu, key < 0 ? -1 : sj);
    const unsigned ga_ = __match_any_sync(0xffffffffu, isang ? sj : -1);
    int pos_r = 0, pos_a = -1;
    if (key >= 0) pos_r = cntw[2 * S + sj] + __popc(gr_ & lt);
    if (isang) pos_a = cntw[3 * S + sj] + __popc(ga_ & lt);
    __syncwarp();
    if (key >= 0 && (gr_ & lt) == 0) cntw[2 * S + sj] += __popc(gr_);
    if (isang && (ga_ & lt) == 0) cntw[3 * S + sj] += __popc(ga_);
    __syncwarp();
    if (k < cnt) {
      float4 v = st.tmp[k];
      float d = sqrtf(fmaxf(v.w, 1e-5f));
      float fc = d < K.rc ? 0.5f * cosf(d * K.pi_rc) + 0.5f : 0.f;
      if (kRd) st.rd[pos_r] = make_float2(d, 0.25f * fc);
      if (kRslot) st.rslot[pos_r] = k;
      if (pos_a >= 0 && pos_a < st.capa) {
        float inv = 1.0f / fmaxf(d, 1e-5f);
        st.au[pos_a] = make_float4(v.x * inv, v.y * inv, v.z * inv, d);
        float sa, ca2;
        sincosf(d * K.pi_rca, &sa, &ca2);
        float fca = d < K.rca ? 0.5f * ca2 + 0.5f : 0.f;
        float dfca = d < K.rca ? -0.5f * K.pi_rca * sa : 0.f;
        st.af[pos_a] = make_float2(fca, dfca);
        if (kGrad) st.aslot[pos_a] = k;
      }
    }
  }
  __syncwarp();
}

// Triangular index t -> (a, b), 0 <= a < b < n, b-major.
__device__ __forceinline__ void tri_ab(int t, int& a, int& b) {
  int bb = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)t)) * 0.5f);
  while (bb * (bb - 1) / 2 > t) --bb;
  while ((bb + 1) * bb / 2 <= t) ++bb;
  b = bb;
  a = t - bb * (bb - 1) / 2;
}

// Diagonal order of the pairs a < b of n items: d = b - a = 1, 2, ...; inside a
// diagonal a increases.  Consecutive t rarely share an item (atomics stay
// nearly conflict-free).
__device__ __forceinline__ void diag_ab(int t, int n, int& a, int& b) {
  float q = (float)(2 * n - 1);
  int u = (int)((q - sqrtf(fmaxf(q * q - 8.0f * (float)t, 0.f))) * 0.5f);
  auto start = [&](int uu) { return (uu * (2 * n - 1) - uu * uu) / 2; };
  while (u > 0 && start(u) > t) --u;
  while (start(u + 1) <= t) ++u;
  a = t - start(u);
  b = a + u + 1;
}

// q = floor(v / n), r = v - q n for 0 <= v < 2^16 and 1 <= n <= 256, from a
// float reciprocal rn = 1/n: (v + 1/2) / n lies at least 1/(2n) from an
// integer, far more than the float error of (v + 1/2) * rn; the correction
// step keeps the result exact even so.
__device__ __forceinline__ void div_small(int v, int n, float rn, int& q, int& r) {
  q = (int)(((float)v + 0.5f) * rn);
  r = v - q * n;
  if (r < 0) {
    --q;
    r += n;
  } else if (r >= n) {
    ++q;
    r -= n;
  }
}

// Reduce v[32] over the warp so that lane f returns sum over lanes of v[f].
__device__ __forceinline__ float transpose_reduce32(float* v, int lane) {
#pragma unroll
  for (int w = 16; w >= 1; w >>= 1) {
    const bool upper = (lane & w) != 0;
#pragma unroll
    for (int k = 0; k < w; ++k) {
      float send = upper ? v[k] : v[k + w];
      float keep = upper ? v[k + w] : v[k];
      v[k] = keep + __shfl_xor_sync(0xffffffffu, send, w);
    }
  }
  return v[0];
}

__device__ __forceinline__ void store_feature(int out_kind, void* out, void* out_lo, size_t idx, float v) {
  if (out_kind == FENNOL_AEV_F32) {
    ((float*)out)[idx] = v;
  } else if (out_kind == FENNOL_AEV_F16X2) {
    const __half hi = __float2half_rn(v);
    ((__half*)out)[idx] = hi;
    ((__half*)out_lo)[idx] = __float2half_rn(v - __half2float(hi));
  } else {
    __nv_bfloat16 hi = to_bf16(v);
    ((__nv_bfloat16*)out)[idx] = hi;
    if (out_kind == FENNOL_AEV_BF16X2) ((__nv_bfloat16*)out_lo)[idx] = to_bf16(v - __bfloat162float(hi));
  }
}

// Asynchronous global -> shared copy of B = 4, 8 or 16 bytes (both addresses
// B-aligned); a thread's copies have landed after cp_async_wait_all.
template <int B>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gmem_src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(gmem_src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Global address of the array that `p` points to in a shared Stage carved at
// dst_base, inside a global record of the same layout at src_base.  Every
// global address is formed from src_base plus the array's offset in the
// layout (a difference of two shared pointers): a pointer computed from a
// shared one would be taken as a shared-window address.
template <typename T>
__device__ __forceinline__ const T* in_record(const char* src_base, const char* dst_base, const T* p) {
  return reinterpret_cast<const T*>(src_base + (reinterpret_cast<const char*>(p) - dst_base));
}

// Warp-collective, asynchronous copy of one centre's staged neighbourhood
// into the shared Stage view `dst` (carved at dst_base) from a global record
// of the same layout (carve_stage(.., cap, false)) at src_base: the cnt
// unsorted edges (vector, d^2, key) and the na angular entries (unit vector
// and d, fc and dfc, row slot).  The forward saves the record for the adjoint
// of the same step, which then skips the gathers and the sort.  Every copy is
// in flight at once; the caller waits (cp_async_wait_all, then __syncwarp).
__device__ __forceinline__ void copy_stage_async(const Stage& dst, const char* dst_base, const char* src_base,
                                                 int cnt, int na, int lane) {
  const float4* tmp = in_record(src_base, dst_base, dst.tmp);
  const int* tkey = in_record(src_base, dst_base, dst.tkey);
  for (int k = lane; k < cnt; k += 32) {
    cp_async<16>(dst.tmp + k, tmp + k);
    cp_async<4>(dst.tkey + k, tkey + k);
  }
  const float4* au = in_record(src_base, dst_base, dst.au);
  const float2* af = in_record(src_base, dst_base, dst.af);
  const int* aslot = in_record(src_base, dst_base, dst.aslot);
  for (int k = lane; k < na; k += 32) {
    cp_async<16>(dst.au + k, au + k);
    cp_async<8>(dst.af + k, af + k);
    cp_async<4>(dst.aslot + k, aslot + k);
  }
}

template <int RD, int AD, int AS, int ZN>
__global__ void __launch_bounds__(kAevWarps * 32)
k_aev_forward(const float4* __restrict__ xyzs, int n, const int* __restrict__ atom_sys,
              const float* __restrict__ sys_cell, const int* __restrict__ nbr_j,
              const unsigned* __restrict__ nbr_shift, const int* __restrict__ nbr_count, int cap,
              const AevConst K, const int* __restrict__ atom_row, int out_kind, void* __restrict__ out,
              void* __restrict__ out_lo, int ld, int* status, char* __restrict__ stage_g) {
  pdl_wait();
  extern __shared__ __align__(16) char smem_c[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kAevWarps + warp;
  if (i >= n) return;
  const int S = K.S;
  Stage st = carve_stage(smem_c + (size_t)warp * stage_bytes(cap), cap);
  const float4 pi = xyzs[i];
  float c[9];
  load_cell(sys_cell, atom_sys[i], c);
  int cnt = nbr_count[i];
  if (cnt > cap) cnt = cap;
  int cnt_r, off_r, cnt_a, off_a, na;
  stage_row<true>(st, st.cntw, xyzs, pi, c, nbr_j, nbr_shift, (size_t)i * cap, cnt, K, lane, cnt_r, off_r, cnt_a,
                  off_a, na);
  if (lane == 0) {
    status_max(status, ST_ANG_MAXCOUNT, na);
    if (na > st.capa) status_set(status, ST_ANG_OVERFLOW);
  }
  if (stage_g) {
    // the saved record uses the adjoint's layout (no sorted radial entries)
    char* rec = stage_g + (size_t)i * stage_bytes(cap, false);
    const Stage rs = carve_stage(rec, cap, false);
    const int nac = min(na, st.capa);
    for (int k = lane; k < cnt; k += 32) {
      rs.tmp[k] = st.tmp[k];
      rs.tkey[k] = st.tkey[k];
    }
    for (int k = lane; k < nac; k += 32) {
      rs.au[k] = st.au[k];
      rs.af[k] = st.af[k];
      rs.aslot[k] = st.aslot[k];
    }
    if (lane < 4 * S) rs.cntw[lane] = st.cntw[lane];
  }
  const size_t orow = (size_t)atom_row[i] * ld;

  // ---- radial: lane (r, h) accumulates feature r over the neighbours h, h+nh, ...
  constexpr int nh = 32 / RD;
  const int r_lane = lane % RD, h_lane = lane / RD;
  const float sr = K.shift_r[r_lane], eta_r = K.eta_r;
  for (int s = 0; s < S; ++s) {
    const int ns = __shfl_sync(0xffffffffu, cnt_r, s);
    const int os = __shfl_sync(0xffffffffu, off_r, s);
    float acc = 0.f;
    for (int t = h_lane; t < ns; t += nh) {
      float2 e = st.rd[os + t];
      float x = e.x - sr;
      acc = fmaf(e.y, fexp(-eta_r * x * x), acc);
    }
    if (nh == 2) acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    if (h_lane == 0) store_feature(out_kind, out, out_lo, orow + s * RD + r_lane, acc);
  }

  // ---- angular: zero every species-pair block, then fill the present ones
  const int FR = S * RD;
  for (int col = lane; col < K.P * 32; col += 32) store_feature(out_kind, out, out_lo, orow + FR + col, 0.f);
  const float c_ang = K.c_ang, eta_a = K.eta_a;
  const unsigned present = __ballot_sync(0xffffffffu, lane < S && cnt_a > 0);
  for (unsigned m1 = present; m1; m1 &= m1 - 1) {
    const int s1 = __ffs(m1) - 1;
    const int n1 = min(__shfl_sync(0xffffffffu, cnt_a, s1), st.capa);
    const int o1 = __shfl_sync(0xffffffffu, off_a, s1);
    for (unsigned m2 = m1; m2; m2 &= m2 - 1) {
      const int s2 = __ffs(m2) - 1;
      const int n2 = min(__shfl_sync(0xffffffffu, cnt_a, s2), st.capa);
      const int o2 = __shfl_sync(0xffffffffu, off_a, s2);
      int T = s1 == s2 ? n1 * (n1 - 1) / 2 : n1 * n2;
      if (o1 + n1 > st.capa || o2 + n2 > st.capa) T = 0;  // overflowing atom: reported above
      if (T == 0) continue;
      const int p = triu_pair(s1, s2, S);
      float acc[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) acc[k] = 0.f;
      for (int t0 = 0; t0 < T; t0 += 32) {
        const int t = t0 + lane;
        if (t < T) {
          int a, b;
          if (s1 == s2) {
            tri_ab(t, a, b);
            a += o1;
            b += o1;
          } else {
            a = o1 + t / n2;
            b = o2 + t % n2;
          }
          const float4 ua = st.au[a], ub = st.au[b];
          const float cosang = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
          const float ct = 0.95f * cosang;
          const float stt = sqrtf(fmaxf(1.0f - ct * ct, 0.f));
          const float f = c_ang * st.af[a].x * st.af[b].x;
          float A[AS], B[AD];
#pragma unroll
          for (int z = 0; z < AS; ++z) {
            float cz = ct * K.cosz[z] + stt * K.sinz[z];
            A[z] = f * zeta_pow<ZN>(1.0f + cz, K.zeta_n, K.zeta_f);
          }
          const float dm = 0.5f * (ua.w + ub.w);
          gauss_chain<AD>(dm - K.shift_a[0], eta_a, K.dra, K.gc2a, B);
#pragma unroll
          for (int r = 0; r < AD; ++r)
#pragma unroll
            for (int z = 0; z < AS; ++z) acc[r * AS + z] = fmaf(A[z], B[r], acc[r * AS + z]);
        }
      }
      const float v = transpose_reduce32(acc, lane);
      __syncwarp();
      store_feature(out_kind, out, out_lo, orow + FR + p * 32 + lane, v);
    }
  }
}

// --------------------------------------------------------------------------------
// Adjoint: dE/dAEV -> forces.
// --------------------------------------------------------------------------------
constexpr int kMaxBlk = kMaxP;  // species-pair blocks of one centre atom

__host__ __device__ __forceinline__ size_t bwd_bytes(int S, int RD, int cap) {
  return (stage_bytes(cap, false) + (size_t)S * (RD + 1) * 4 + (6 * kMaxBlk + 2) * 4 + 15) / 16 * 16;
}

template <int RD, int AD, int AS, int ZN, bool kVir, bool kStaged>
__global__ void __launch_bounds__(kAevWarps * 32, 4)
k_aev_backward(const float4* __restrict__ xyzs, int n, const int* __restrict__ atom_sys,
               const float* __restrict__ sys_cell, const int* __restrict__ nbr_j,
               const unsigned* __restrict__ nbr_shift, const int* __restrict__ nbr_count, int cap,
               const AevConst K, const int* __restrict__ atom_row, const float* __restrict__ daev,
               int ld, float4* __restrict__ forces, float* __restrict__ atom_virial, int* status,
               const char* __restrict__ stage_g) {
  pdl_wait();
  extern __shared__ __align__(16) char smem_c[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kAevWarps + warp;
  if (i >= n) return;
  const int S = K.S;
  char* base = smem_c + (size_t)warp * bwd_bytes(S, RD, cap);
  Stage st = carve_stage(base, cap, false);
  // the edge vectors in st.tmp[k] are replaced by the gradient of the energy
  // with respect to edge k (x, y, z) once the radial pass has read them
  float* gk = reinterpret_cast<float*>(st.tmp);
  float* gr = (float*)(base + stage_bytes(cap, false));               // [S][RD+1]
  int* blkw = (int*)(gr + S * (RD + 1));                              // block table

  // Two dependent rounds of global loads: the row index, row length and
  // (staged) the per-species counters, then every copy of the dE/dAEV row and
  // of the staged record at once, as asynchronous copies into shared memory.
  const int arow = atom_row[i];
  int cnt = nbr_count[i];
  const char* rec = nullptr;
  int cw = 0;
  if constexpr (kStaged) {
    // the forward of this step staged this centre already
    rec = stage_g + (size_t)i * stage_bytes(cap, false);
    if (lane < 4 * S) cw = in_record(rec, base, st.cntw)[lane];
  }
  const float* g = daev + (size_t)arow * ld;
  const int FR = S * RD;
  for (int col = lane; col < FR; col += 32) cp_async<4>(gr + (col / RD) * (RD + 1) + col % RD, g + col);
  const float4 pi = xyzs[i];
  float c[9];
  load_cell(sys_cell, atom_sys[i], c);
  if (cnt > cap) cnt = cap;
  const size_t row = (size_t)i * cap;
  if constexpr (kStaged) {
    if (lane < 4 * S) st.cntw[lane] = cw;
    int na = lane >= S && lane < 2 * S ? cw : 0;  // angular counts per species
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) na += __shfl_xor_sync(0xffffffffu, na, o);
    copy_stage_async(st, base, rec, cnt, min(na, st.capa), lane);
    cp_async_wait_all();
    __syncwarp();
  } else {
    int cnt_r, off_r, cnt_a, off_a, na;
    stage_row<true, false, false>(st, st.cntw, xyzs, pi, c, nbr_j, nbr_shift, row, cnt, K, lane, cnt_r, off_r,
                                  cnt_a, off_a, na);
    if (na > st.capa && lane == 0) status_set(status, ST_ANG_OVERFLOW);
    cp_async_wait_all();
    __syncwarp();
  }

  // ---- radial: lane per neighbour (row order), gradient into gk[4k..4k+2]
  for (int k = lane; k < cnt; k += 32) {
    const float4 v = st.tmp[k];
    const int sj = st.tkey[k] & 0xFF;
    const float d = sqrtf(fmaxf(v.w, 1e-5f));
    float fc = 0.f, dfc = 0.f;
    if (d < K.rc) {
      float sa, ca;
      sincosf(d * K.pi_rc, &sa, &ca);
      fc = 0.5f * ca + 0.5f;
      dfc = -0.5f * K.pi_rc * sa;
    }
    const float* grow = gr + sj * (RD + 1);
    float dEdd = 0.f;
    float Br[RD];
    gauss_chain_from<RD>(d - K.shift_r[0], K.eta_r, K.drr, K.inv_drr, K.gc2r, K.lim_r, Br);
#pragma unroll
    for (int r = 0; r < RD; ++r) {
      float x = d - K.shift_r[r];
      dEdd = fmaf(grow[r] * Br[r], dfc - 2.f * K.eta_r * x * fc, dEdd);
    }
    float sc = v.w > 1e-5f ? 0.25f * dEdd / d : 0.f;
    st.tmp[k] = make_float4(sc * v.x, sc * v.y, sc * v.z, 0.f);
  }
  __syncwarp();

  // ---- angular: the triplets of all present species-pair blocks are packed
  // into consecutive warp rounds (lane per triplet); each lane reads the
  // dE/dAEV row of its own pair block.
  const float zeta = K.zeta, c_ang = K.c_ang, eta_a = K.eta_a, zm1 = K.zeta - 1.0f;
  // Block table, built once per centre so that a triplet needs no per-species
  // lookups: first triplet, sizes, offsets, pair index, 1/n of each block.
  int* blk_cum = blkw;                                   // [kMaxBlk + 2]: first triplet, end, count
  int* blk_n = blkw + kMaxBlk + 2;                       // n1 | n2 << 12 | (s1 == s2) << 24
  int* blk_o = blk_n + kMaxBlk;                          // o1 | o2 << 12 (counts and offsets <= 256)
  int* blk_p = blk_o + kMaxBlk;                          // species-pair index
  float* blk_r1 = reinterpret_cast<float*>(blk_p + kMaxBlk);  // 1 / n1
  float* blk_r2 = blk_r1 + kMaxBlk;                           // 1 / n2
  // Lane l of round q takes the species pair (s1, s2) = divmod(32 q + l, S),
  // kept when s1 <= s2: lane order is the s1-major order of the blocks.  A
  // ballot numbers the non-empty blocks and a warp scan accumulates their
  // first triplets.
  {
    int nb = 0, tot = 0;
    for (int l0 = 0; l0 < S * S; l0 += 32) {
      const int l = l0 + lane;
      const int s1 = l / S, s2 = l - (l / S) * S;
      int T = 0, n1 = 0, n2 = 0, o1 = 0, o2 = 0;
      if (l < S * S && s1 <= s2) {
        n1 = min(st.cntw[S + s1], st.capa);
        n2 = min(st.cntw[S + s2], st.capa);
        o1 = st.cntw[3 * S + s1] - st.cntw[S + s1];  // running offset ended at off + count
        o2 = st.cntw[3 * S + s2] - st.cntw[S + s2];
        T = s1 == s2 ? n1 * (n1 - 1) / 2 : n1 * n2;
        if (o1 + n1 > st.capa || o2 + n2 > st.capa) T = 0;
      }
      const unsigned has = __ballot_sync(0xffffffffu, T > 0);
      int incl = T;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (T > 0) {
        const int k = nb + __popc(has & ((1u << lane) - 1u));
        blk_cum[k] = tot + incl - T;
        blk_n[k] = n1 | (n2 << 12) | ((s1 == s2) << 24);
        blk_o[k] = o1 | (o2 << 12);
        blk_p[k] = triu_pair(s1, s2, S);
        blk_r1[k] = 1.0f / (float)n1;
        blk_r2[k] = 1.0f / (float)n2;
      }
      nb += __popc(has);
      tot += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) {
      blk_cum[nb] = tot;
      blk_cum[kMaxBlk + 1] = nb;
    }
  }
  __syncwarp();
  const int nblk = blk_cum[kMaxBlk + 1];
  const int Ttot = blk_cum[nblk];
  for (int t = lane; t < Ttot; t += 32) {
    int k = 0;
    while (k + 1 < nblk && blk_cum[k + 1] <= t) ++k;
    const int tl = t - blk_cum[k];
    const int nn = blk_n[k], oo = blk_o[k];
    const int n1 = nn & 0xFFF, n2 = (nn >> 12) & 0xFFF;
    const int o1 = oo & 0xFFF, o2 = oo >> 12;
    int a, b;
    if (nn >> 24) {
      diag_ab(tl, n1, a, b);
      a += o1;
      b += o1;
    } else {
      // aa = tl mod n1, dd = tl div n1, b = o2 + (aa + dd) mod n2, as exact
      // quotients through 1/n (n <= 256, tl < 256 * 256)
      int dd, aa, bb;
      div_small(tl, n1, blk_r1[k], dd, aa);
      int q2;
      div_small(aa + dd, n2, blk_r2[k], q2, bb);
      a = o1 + aa;
      b = o2 + bb;
    }
    const int p = blk_p[k];
    const float* gp = g + FR + p * 32;
    const float4 ua = st.au[a], ub = st.au[b];
    const float2 fa2 = st.af[a], fb2 = st.af[b];
    const float cosang = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
    const float ct = 0.95f * cosang;
    const float stt = sqrtf(fmaxf(1.0f - ct * ct, 1e-12f));
    float A[AS], Ap[AS];
#pragma unroll
    for (int z = 0; z < AS; ++z) {
      float cz = ct * K.cosz[z] + stt * K.sinz[z];
      float sz = stt * K.cosz[z] - ct * K.sinz[z];
      float bs = fmaxf(1.0f + cz, 0.f);
      // (1 + cz)^(zeta - 1) from one SFU log2 and exp2: ~2e-6 relative error
      // (the log2 error scaled by zeta - 1), negligible in a force term
      const float pw1 = bs > 0.f ? exp2f_approx_pos(zm1 * __log2f(bs)) : 0.f;
      A[z] = pw1 * bs;
      Ap[z] = -zeta * pw1 * sz;
    }
    const float dm = 0.5f * (ua.w + ub.w);
    float Q = 0.f, Th = 0.f, Dm = 0.f;
    float Bs[AD];
    gauss_chain<AD>(dm - K.shift_a[0], eta_a, K.dra, K.gc2a, Bs);
#pragma unroll
    for (int r = 0; r < AD; ++r) {
      const float x = dm - K.shift_a[r];
      const float Bv = Bs[r];
      float GA = 0.f, GAp = 0.f;
      // the pair block (32 floats) starts 16-byte aligned when ld and S * RD
      // are multiples of 4 (checked by the launcher)
      float gz[AS];
#pragma unroll
      for (int z4 = 0; z4 < AS / 4; ++z4) {
        const float4 q = __ldg(reinterpret_cast<const float4*>(gp + r * AS) + z4);
        gz[4 * z4] = q.x;
        gz[4 * z4 + 1] = q.y;
        gz[4 * z4 + 2] = q.z;
        gz[4 * z4 + 3] = q.w;
      }
#pragma unroll
      for (int z = 0; z < AS; ++z) {
        GA = fmaf(gz[z], A[z], GA);
        GAp = fmaf(gz[z], Ap[z], GAp);
      }
      Q = fmaf(GA, Bv, Q);
      Th = fmaf(GAp, Bv, Th);
      Dm = fmaf(GA, -2.f * eta_a * x * Bv, Dm);
    }
    const float fa = fa2.x, fb = fb2.x;
    const float cfab = c_ang * fa * fb;
    const float dEddm = cfab * Dm;
    const float dEdda = 0.5f * dEddm + c_ang * fb * Q * fa2.y;
    const float dEddb = 0.5f * dEddm + c_ang * fa * Q * fb2.y;
    const float dEdc = cfab * Th * (-0.95f * rsqrtf(fmaxf(1.0f - ct * ct, 1e-12f)));
    const float ia = __fdividef(dEdc, ua.w), ib = __fdividef(dEdc, ub.w);
    const int sa_ = st.aslot[a], sb_ = st.aslot[b];
    atomicAdd(gk + 4 * sa_, dEdda * ua.x + ia * (ub.x - cosang * ua.x));
    atomicAdd(gk + 4 * sa_ + 1, dEdda * ua.y + ia * (ub.y - cosang * ua.y));
    atomicAdd(gk + 4 * sa_ + 2, dEdda * ua.z + ia * (ub.z - cosang * ua.z));
    atomicAdd(gk + 4 * sb_, dEddb * ub.x + ib * (ua.x - cosang * ub.x));
    atomicAdd(gk + 4 * sb_ + 1, dEddb * ub.y + ib * (ua.y - cosang * ub.y));
    atomicAdd(gk + 4 * sb_ + 2, dEddb * ub.z + ib * (ua.z - cosang * ub.z));
  }
  __syncwarp();

  // ---- scatter: F_j -= g, F_i += sum g
  float fx = 0.f, fy = 0.f, fz = 0.f;
  for (int k = lane; k < cnt; k += 32) {
    const float4 gv = st.tmp[k];
    const float gx = gv.x, gy = gv.y, gz = gv.z;
    int j = __ldg(nbr_j + row + k);
    atomicAdd(forces + j, make_float4(-gx, -gy, -gz, 0.f));
    fx += gx;
    fy += gy;
    fz += gz;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
  }
  if (lane == 0) atomicAdd(forces + i, make_float4(fx, fy, fz, 0.f));

  // ---- virial of this centre: sum over its edges of r (x) dE/dr
  if (kVir) {
    float v[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) v[q] = 0.f;
    for (int k = lane; k < cnt; k += 32) {
      const float4 gv = st.tmp[k];
      float rx, ry, rz;
      edge_vec(pi, xyzs[__ldg(nbr_j + row + k)], __ldg(nbr_shift + row + k), c, rx, ry, rz);
      v[0] = fmaf(rx, gv.x, v[0]);
      v[1] = fmaf(rx, gv.y, v[1]);
      v[2] = fmaf(rx, gv.z, v[2]);
      v[3] = fmaf(ry, gv.x, v[3]);
      v[4] = fmaf(ry, gv.y, v[4]);
      v[5] = fmaf(ry, gv.z, v[5]);
      v[6] = fmaf(rz, gv.x, v[6]);
      v[7] = fmaf(rz, gv.y, v[7]);
      v[8] = fmaf(rz, gv.z, v[8]);
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    if (lane < 9) {
      float out = v[0];
#pragma unroll
      for (int q = 1; q < 9; ++q) out = lane == q ? v[q] : out;
      atom_virial[(size_t)i * 9 + lane] = out;
    }
  }
}

// --------------------------------------------------------------------------------
// Tangent (forward mode): t = dAEV/dx . u for a displacement field u.  With
// F = -dE/dx, the force term of a training loss differentiates
// sum_i <dE/dAEV_i, t_i> with respect to the network parameters, which needs
// the AEV tangent along u = dL/dF (the second-order term of jax.grad over a
// force loss, training/utils.py:140-525).
// --------------------------------------------------------------------------------
__host__ __device__ __forceinline__ size_t jvp_bytes(int cap) {
  return (stage_bytes(cap) + (size_t)cap * (4 + 16 + 8) + 15) / 16 * 16;
}

template <int RD, int AD, int AS, int ZN>
__global__ void __launch_bounds__(kAevWarps * 32)
k_aev_tangent(const float4* __restrict__ xyzs, int n, const int* __restrict__ atom_sys,
              const float* __restrict__ sys_cell, const int* __restrict__ nbr_j,
              const unsigned* __restrict__ nbr_shift, const int* __restrict__ nbr_count, int cap,
              const AevConst K, const int* __restrict__ atom_row, const float4* __restrict__ du,
              float* __restrict__ out, int ld, int* status) {
  pdl_wait();
  extern __shared__ __align__(16) char smem_c[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kAevWarps + warp;
  if (i >= n) return;
  const int S = K.S;
  char* base = smem_c + (size_t)warp * jvp_bytes(cap);
  Stage st = carve_stage(base, cap);
  float4* tanw = (float4*)(base + stage_bytes(cap));  // [cap] (u_j - u_i) / d, d-dot (row order)
  float2* tanr = (float2*)(tanw + cap);                // [cap] d-dot, 0.25 fc'(d)  (row order)
  st.rslot = (int*)(tanr + cap);                       // [cap]
  const float4 pi = xyzs[i];
  const float4 ui = du[i];
  float c[9];
  load_cell(sys_cell, atom_sys[i], c);
  int cnt = nbr_count[i];
  if (cnt > cap) cnt = cap;
  const size_t row = (size_t)i * cap;
  int cnt_r, off_r, cnt_a, off_a, na;
  stage_row<true, true>(st, st.cntw, xyzs, pi, c, nbr_j, nbr_shift, row, cnt, K, lane, cnt_r, off_r, cnt_a,
                        off_a, na);
  if (na > st.capa && lane == 0) status_set(status, ST_ANG_OVERFLOW);

  // per-neighbour tangents: d-dot = r.(u_j - u_i)/d and (u_j - u_i)/d
  for (int k = lane; k < cnt; k += 32) {
    const float4 v = st.tmp[k];
    const float4 uj = du[__ldg(nbr_j + row + k)];
    const float rx = uj.x - ui.x, ry = uj.y - ui.y, rz = uj.z - ui.z;
    const float d = sqrtf(fmaxf(v.w, 1e-5f));
    const float inv = v.w > 1e-5f ? 1.0f / d : 0.f;  // safe_sqrt clip: no tangent below it
    const float dd = (v.x * rx + v.y * ry + v.z * rz) * inv;
    tanw[k] = make_float4(rx * inv, ry * inv, rz * inv, dd);
    const float dfc = d < K.rc ? -0.5f * K.pi_rc * sinf(d * K.pi_rc) : 0.f;
    tanr[k] = make_float2(dd, 0.25f * dfc);
  }
  __syncwarp();
  const size_t orow = (size_t)atom_row[i] * ld;

  // ---- radial: d/dt [0.25 fc(d) exp(-eta (d - R)^2)]
  constexpr int nh = 32 / RD;
  const int r_lane = lane % RD, h_lane = lane / RD;
  const float sr = K.shift_r[r_lane], eta_r = K.eta_r;
  for (int s = 0; s < S; ++s) {
    const int ns = __shfl_sync(0xffffffffu, cnt_r, s);
    const int os = __shfl_sync(0xffffffffu, off_r, s);
    float acc = 0.f;
    for (int t = h_lane; t < ns; t += nh) {
      const float2 e = st.rd[os + t];
      const float2 tr = tanr[st.rslot[os + t]];
      const float x = e.x - sr;
      acc = fmaf(fexp(-eta_r * x * x) * (tr.y - 2.f * eta_r * x * e.y), tr.x, acc);
    }
    if (nh == 2) acc += __shfl_xor_sync(0xffffffffu, acc, 16);
    if (h_lane == 0) out[orow + s * RD + r_lane] = acc;
  }

  // ---- angular
  const int FR = S * RD;
  for (int col = lane; col < K.P * 32; col += 32) out[orow + FR + col] = 0.f;
  const float c_ang = K.c_ang, eta_a = K.eta_a, zeta = K.zeta;
  const unsigned present = __ballot_sync(0xffffffffu, lane < S && cnt_a > 0);
  for (unsigned m1 = present; m1; m1 &= m1 - 1) {
    const int s1 = __ffs(m1) - 1;
    const int n1 = min(__shfl_sync(0xffffffffu, cnt_a, s1), st.capa);
    const int o1 = __shfl_sync(0xffffffffu, off_a, s1);
    for (unsigned m2 = m1; m2; m2 &= m2 - 1) {
      const int s2 = __ffs(m2) - 1;
      const int n2 = min(__shfl_sync(0xffffffffu, cnt_a, s2), st.capa);
      const int o2 = __shfl_sync(0xffffffffu, off_a, s2);
      int T = s1 == s2 ? n1 * (n1 - 1) / 2 : n1 * n2;
      if (o1 + n1 > st.capa || o2 + n2 > st.capa) T = 0;
      if (T == 0) continue;
      const int p = triu_pair(s1, s2, S);
      float acc[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) acc[k] = 0.f;
      for (int t0 = 0; t0 < T; t0 += 32) {
        const int t = t0 + lane;
        if (t < T) {
          int a, b;
          if (s1 == s2) {
            tri_ab(t, a, b);
            a += o1;
            b += o1;
          } else {
            a = o1 + t / n2;
            b = o2 + t % n2;
          }
          const float4 ua = st.au[a], ub = st.au[b];
          const float2 fa = st.af[a], fb = st.af[b];
          const float4 wa = tanw[st.aslot[a]], wb = tanw[st.aslot[b]];
          const float cosang = ua.x * ub.x + ua.y * ub.y + ua.z * ub.z;
          // d/dt of u_a . u_b with u = r / |r|
          const float dcos = (wa.x * ub.x + wa.y * ub.y + wa.z * ub.z) - cosang * wa.w / ua.w +
                             (wb.x * ua.x + wb.y * ua.y + wb.z * ua.z) - cosang * wb.w / ub.w;
          const float ct = 0.95f * cosang, dct = 0.95f * dcos;
          const float stt = sqrtf(fmaxf(1.0f - ct * ct, 1e-12f));
          const float dstt = -ct * dct / stt;
          const float f = c_ang * fa.x * fb.x;
          const float df = c_ang * (fa.y * wa.w * fb.x + fa.x * fb.y * wb.w);
          float A[AS], dA[AS];
#pragma unroll
          for (int z = 0; z < AS; ++z) {
            const float cz = ct * K.cosz[z] + stt * K.sinz[z];
            const float dcz = dct * K.cosz[z] + dstt * K.sinz[z];
            const float bs = fmaxf(1.0f + cz, 0.f);
            const float pw1 = zeta_pow<zn_minus1(ZN)>(bs, K.zeta1_n, K.zeta1_f);  // (1 + cz)^(zeta - 1)
            A[z] = f * pw1 * bs;
            dA[z] = df * pw1 * bs + f * zeta * pw1 * dcz;
          }
          const float dm = 0.5f * (ua.w + ub.w), ddm = 0.5f * (wa.w + wb.w);
          float Bs[AD];
          gauss_chain<AD>(dm - K.shift_a[0], eta_a, K.dra, K.gc2a, Bs);
#pragma unroll
          for (int r = 0; r < AD; ++r) {
            const float x = dm - K.shift_a[r];
            const float B = Bs[r];
            const float dB = -2.f * eta_a * x * ddm * B;
#pragma unroll
            for (int z = 0; z < AS; ++z) acc[r * AS + z] = fmaf(dA[z], B, fmaf(A[z], dB, acc[r * AS + z]));
          }
        }
      }
      const float v = transpose_reduce32(acc, lane);
      __syncwarp();
      out[orow + FR + p * 32 + lane] = v;
    }
  }
}


__global__ void k_pack(const float* __restrict__ coords, const int* __restrict__ sp, int n,
                       float4* __restrict__ xyzs) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xyzs[i] = make_float4(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], __int_as_float(sp[i]));
}

template <int RD, int AD, int AS, int ZN>
struct AevKernels {
  static constexpr auto fwd = k_aev_forward<RD, AD, AS, ZN>;
  static constexpr auto bwd = k_aev_backward<RD, AD, AS, ZN, false, false>;
  static constexpr auto bwdv = k_aev_backward<RD, AD, AS, ZN, true, false>;
  static constexpr auto bwds = k_aev_backward<RD, AD, AS, ZN, false, true>;
  static constexpr auto tan = k_aev_tangent<RD, AD, AS, ZN>;
};

// (RD, AD, AS) combinations compiled: radial 16/32 x angular (8,4) / (4,8),
// with the integer part of zeta read at run time; the ANI-2x layout
// (16 radial shifts, 8 angular shifts x 4 sections) with zeta in [14, 15)
// also has kernels with it built in.
template <typename Fn>
bool dispatch(const AevConst& K, Fn&& fn) {
  if (K.RD == 16 && K.AD == 8 && K.AS == 4 && K.zeta_n == 14) return fn(AevKernels<16, 8, 4, 14>{});
  if (K.RD == 16 && K.AD == 8 && K.AS == 4) return fn(AevKernels<16, 8, 4, -1>{});
  if (K.RD == 16 && K.AD == 4 && K.AS == 8) return fn(AevKernels<16, 4, 8, -1>{});
  if (K.RD == 32 && K.AD == 8 && K.AS == 4) return fn(AevKernels<32, 8, 4, -1>{});
  if (K.RD == 32 && K.AD == 4 && K.AS == 8) return fn(AevKernels<32, 4, 8, -1>{});
  return false;
}

// Opt a kernel in to the largest dynamic shared memory it can use, once.
size_t set_smem(const void* fn, size_t bytes) {
  static const void* done[32] = {};
  if (bytes > 48 * 1024) {
    for (int k = 0; k < 32; ++k) {
      if (done[k] == fn) return bytes;
      if (!done[k]) {
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024) != cudaSuccess)
          return 0;
        done[k] = fn;
        return bytes;
      }
    }
    return 0;
  }
  return bytes;
}

}  // namespace

extern "C" int fennol_aev_length(const fennol_aev_params* p) {
  AevConst k;
  if (!make_const(p, &k)) return -1;
  return k.F;
}

extern "C" unsigned long long fennol_aev_active_chunks(const fennol_aev_params* p, unsigned species_mask) {
  if (fennol_aev_length(p) <= 0) return 0ull;
  const int S = p->num_species, RD = p->radial_divisions;
  const int A = p->angular_divisions * p->angle_sections;
  const int F = S * RD + S * (S + 1) / 2 * A;
  if (F > 64 * 64) return 0ull;
  unsigned long long m = 0ull;
  auto mark = [&](int c0, int c1) {  // columns [c0, c1)
    for (int c = c0 / 64; c <= (c1 - 1) / 64; ++c) m |= 1ull << c;
  };
  for (int s = 0; s < S; ++s)
    if ((species_mask >> s) & 1u) mark(s * RD, (s + 1) * RD);
  for (int s1 = 0; s1 < S; ++s1)
    for (int s2 = s1; s2 < S; ++s2)
      if (((species_mask >> s1) & 1u) && ((species_mask >> s2) & 1u)) {
        const int c0 = S * RD + fnl::triu_pair(s1, s2, S) * A;
        mark(c0, c0 + A);
      }
  return m;
}

extern "C" int fennol_pack_atoms(const float* coords, const int* species_idx, int natoms, float* xyzs,
                                 void* stream) {
  if (natoms < 0 || (natoms > 0 && (!coords || !species_idx || !xyzs))) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  FNL_LAUNCH_PDL(k_pack, (natoms + 255) / 256, 256, 0, (cudaStream_t)stream, coords, species_idx, natoms,
                                                                  (float4*)xyzs);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

static int aev_forward_launch(const float* xyzs, int natoms, const int* atom_sys, const float* sys_cell,
                              const int* nbr_j, const unsigned* nbr_shift, const int* nbr_count, int capacity,
                              const fennol_aev_params* p, const int* atom_row, int out_kind, void* out,
                              void* out_lo, int ld, int* status, void* stage, void* stream) {
  AevConst K;
  if (!make_const(p, &K)) return FENNOL_ERR_UNSUPPORTED;
  if (natoms < 0 || capacity <= 0 || ld < K.F) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!xyzs || !atom_sys || !nbr_j || !nbr_shift || !nbr_count || !atom_row || !out)
    return FENNOL_ERR_INVALID;
  if (out_kind != FENNOL_AEV_F32 && out_kind != FENNOL_AEV_BF16 && out_kind != FENNOL_AEV_BF16X2 &&
      out_kind != FENNOL_AEV_F16X2)
    return FENNOL_ERR_INVALID;
  if ((out_kind == FENNOL_AEV_BF16X2 || out_kind == FENNOL_AEV_F16X2) && !out_lo) return FENNOL_ERR_INVALID;
  if ((size_t)kAevWarps * stage_bytes(capacity) > 200 * 1024) return FENNOL_ERR_UNSUPPORTED;
  int blocks = (natoms + kAevWarps - 1) / kAevWarps;
  bool launched = dispatch(K, [&](auto ks) {
    size_t smem = set_smem((const void*)ks.fwd, (size_t)kAevWarps * stage_bytes(capacity));
    if (!smem) return false;
    if (launch_pdl(ks.fwd, blocks, kAevWarps * 32, smem, (cudaStream_t)stream, 
        (const float4*)xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, K,
        atom_row, out_kind, out, out_lo, ld, status, (char*)stage) != cudaSuccess) return false;
    return true;
  });
  if (!launched) return FENNOL_ERR_UNSUPPORTED;
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_aev_forward(const float* xyzs, int natoms, const int* atom_sys,
                                  const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                  const int* nbr_count, int capacity, const fennol_aev_params* p,
                                  const int* atom_row, int out_kind, void* out, void* out_lo, int ld,
                                  int* status, void* stream) {
  return aev_forward_launch(xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, p, atom_row,
                            out_kind, out, out_lo, ld, status, nullptr, stream);
}

extern "C" size_t fennol_aev_stage_bytes(int natoms, int capacity) {
  if (natoms < 0 || capacity <= 0) return 0;
  return (size_t)natoms * stage_bytes(capacity, false);
}

extern "C" int fennol_aev_forward_staged(const float* xyzs, int natoms, const int* atom_sys,
                                         const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                         const int* nbr_count, int capacity, const fennol_aev_params* p,
                                         const int* atom_row, int out_kind, void* out, void* out_lo, int ld,
                                         void* stage, size_t stage_bytes_, int* status, void* stream) {
  if (natoms > 0 && (!stage || ((uintptr_t)stage & 15) != 0)) return FENNOL_ERR_INVALID;
  if (stage_bytes_ < fennol_aev_stage_bytes(natoms, capacity)) return FENNOL_ERR_WORKSPACE;
  return aev_forward_launch(xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, p, atom_row,
                            out_kind, out, out_lo, ld, status, stage, stream);
}

static int aev_backward_launch(const float* xyzs, int natoms, const int* atom_sys, const float* sys_cell,
                               const int* nbr_j, const unsigned* nbr_shift, const int* nbr_count, int capacity,
                               const fennol_aev_params* p, const int* atom_row, const float* daev, int ld,
                               float* forces4, float* atom_virial, int* status, const void* stage,
                               void* stream) {
  AevConst K;
  if (!make_const(p, &K)) return FENNOL_ERR_UNSUPPORTED;
  if (natoms < 0 || capacity <= 0 || ld < K.F) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!xyzs || !atom_sys || !nbr_j || !nbr_shift || !nbr_count || !atom_row || !daev || !forces4)
    return FENNOL_ERR_INVALID;
  // the kernel reads dE/dAEV pair blocks as float4
  if ((ld & 3) != 0 || ((uintptr_t)daev & 15) != 0) return FENNOL_ERR_INVALID;
  size_t bytes = (size_t)kAevWarps * bwd_bytes(K.S, K.RD, capacity);
  if (bytes > 200 * 1024) return FENNOL_ERR_UNSUPPORTED;
  int blocks = (natoms + kAevWarps - 1) / kAevWarps;
  bool launched = dispatch(K, [&](auto ks) {
    auto fn = atom_virial ? ks.bwdv : (stage ? ks.bwds : ks.bwd);
    size_t smem = set_smem((const void*)fn, bytes);
    if (!smem) return false;
    if (launch_pdl(fn, blocks, kAevWarps * 32, smem, (cudaStream_t)stream, 
        (const float4*)xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, K,
        atom_row, daev, ld, (float4*)forces4, atom_virial, status, (const char*)stage) != cudaSuccess) return false;
    return true;
  });
  if (!launched) return FENNOL_ERR_UNSUPPORTED;
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_aev_backward(const float* xyzs, int natoms, const int* atom_sys,
                                   const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                   const int* nbr_count, int capacity, const fennol_aev_params* p,
                                   const int* atom_row, const float* daev, int ld, float* forces4,
                                   int* status, void* stream) {
  return aev_backward_launch(xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, p,
                             atom_row, daev, ld, forces4, nullptr, status, nullptr, stream);
}

extern "C" int fennol_aev_backward_staged(const float* xyzs, int natoms, const int* atom_sys,
                                          const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                          const int* nbr_count, int capacity, const fennol_aev_params* p,
                                          const int* atom_row, const float* daev, int ld, float* forces4,
                                          const void* stage, int* status, void* stream) {
  if (natoms > 0 && (!stage || ((uintptr_t)stage & 15) != 0)) return FENNOL_ERR_INVALID;
  return aev_backward_launch(xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, p,
                             atom_row, daev, ld, forces4, nullptr, status, stage, stream);
}

extern "C" int fennol_aev_backward_virial(const float* xyzs, int natoms, const int* atom_sys,
                                          const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                          const int* nbr_count, int capacity, const fennol_aev_params* p,
                                          const int* atom_row, const float* daev, int ld, float* forces4,
                                          float* atom_virial, int* status, void* stream) {
  if (natoms > 0 && !atom_virial) return FENNOL_ERR_INVALID;
  return aev_backward_launch(xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, p,
                             atom_row, daev, ld, forces4, atom_virial, status, nullptr, stream);
}

extern "C" int fennol_aev_tangent(const float* xyzs, int natoms, const int* atom_sys,
                                  const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                  const int* nbr_count, int capacity, const fennol_aev_params* p,
                                  const int* atom_row, const float* du4, float* out, int ld, int* status,
                                  void* stream) {
  AevConst K;
  if (!make_const(p, &K)) return FENNOL_ERR_UNSUPPORTED;
  if (natoms < 0 || capacity <= 0 || ld < K.F) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!xyzs || !atom_sys || !nbr_j || !nbr_shift || !nbr_count || !atom_row || !du4 || !out)
    return FENNOL_ERR_INVALID;
  size_t bytes = (size_t)kAevWarps * jvp_bytes(capacity);
  if (bytes > 200 * 1024) return FENNOL_ERR_UNSUPPORTED;
  int blocks = (natoms + kAevWarps - 1) / kAevWarps;
  bool launched = dispatch(K, [&](auto ks) {
    size_t smem = set_smem((const void*)ks.tan, bytes);
    if (!smem) return false;
    if (launch_pdl(ks.tan, blocks, kAevWarps * 32, smem, (cudaStream_t)stream, 
        (const float4*)xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, K,
        atom_row, (const float4*)du4, out, ld, status) != cudaSuccess) return false;
    return true;
  });
  if (!launched) return FENNOL_ERR_UNSUPPORTED;
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}
