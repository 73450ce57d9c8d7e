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

constexpr int kAevWarps = 4;
constexpr int kMaxS = 8;
constexpr int kMaxP = kMaxS * (kMaxS + 1) / 2;
constexpr int kCapA = FENNOL_MAX_ANGULAR_NEIGHBORS;
constexpr float kPi = 3.14159265358979323846f;

struct AevConst {
  int S, P, RD, AD, AS, F;
  float rc, rca, rc2, rca2;   // cutoffs and float32 thresholds
  float pi_rc, pi_rca;        // pi / cutoff
  float eta_r, eta_a, zeta, c_ang;  // c_ang = 2^(1-zeta)
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
  for (int r = 0; r < 32; ++r) {
    k->shift_r[r] = r < RD ? (float)(p->radial_start + (p->radial_cutoff - p->radial_start) * r / RD) : 0.f;
    k->shift_a[r] = r < AD ? (float)(p->angular_start + (p->angular_cutoff - p->angular_start) * r / AD) : 0.f;
    double z = M_PI * r / AS + M_PI / (2.0 * AS);
    k->cosz[r] = r < AS ? (float)std::cos(z) : 0.f;
    k->sinz[r] = r < AS ? (float)std::sin(z) : 0.f;
  }
  return true;
}

// Triplet index t -> (a, b) with a < b, enumerated b = 1.., a = 0..b-1.
__device__ __forceinline__ void triplet_ab(int t, int& a, int& b) {
  int bb = (int)((1.0f + sqrtf(1.0f + 8.0f * (float)t)) * 0.5f);
  while (bb * (bb - 1) / 2 > t) --bb;
  while ((bb + 1) * bb / 2 <= t) ++bb;
  b = bb;
  a = t - bb * (bb - 1) / 2;
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

// Shared-memory carve-up per warp (floats).
struct FwdSmem {
  float* rad;    // [S][32]
  float* ang;    // [P][32]
  float* au;     // [kCapA][4] ux,uy,uz,d
  float* afc;    // [kCapA]
  int* asp;      // [kCapA]
  float* stA;    // [32][33] angular factors (scaled by the switch product)
  float* stB;    // [32][33] radial factors
  int* stP;      // [32]
};
__host__ __device__ __forceinline__ int fwd_smem_floats(int S, int P) {
  return S * 32 + P * 32 + kCapA * 6 + 32 * 33 + 32 * 33 + 32;
}

template <int RD, int AD, int AS>
__global__ void __launch_bounds__(kAevWarps * 32)
k_aev_forward(const float4* __restrict__ xyzs, int n, const int* __restrict__ atom_sys,
              const float* __restrict__ sys_cell, const int* __restrict__ nbr_j,
              const unsigned* __restrict__ nbr_shift, const int* __restrict__ nbr_count, int cap,
              const AevConst K, const int* __restrict__ atom_row, int out_kind, void* __restrict__ out,
              void* __restrict__ out_lo, int ld, int* status) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kAevWarps + warp;
  if (i >= n) return;
  const int S = K.S, P = K.P;
  float* base = smem + (size_t)warp * fwd_smem_floats(S, P);
  FwdSmem sm;
  sm.rad = base;
  sm.ang = sm.rad + S * 32;
  sm.au = sm.ang + P * 32;
  sm.afc = sm.au + kCapA * 4;
  sm.asp = (int*)(sm.afc + kCapA);
  sm.stA = (float*)(sm.asp + kCapA);
  sm.stB = sm.stA + 32 * 33;
  sm.stP = (int*)(sm.stB + 32 * 33);

  for (int k = lane; k < (S + P) * 32; k += 32) sm.rad[k] = 0.f;
  __syncwarp();

  const float4 pi = xyzs[i];
  float c[9];
  load_cell(sys_cell, atom_sys[i], c);
  int cnt = nbr_count[i];
  if (cnt > cap) cnt = cap;
  const size_t row = (size_t)i * cap;
  constexpr int nh = 32 / RD;    // neighbours per radial step
  const int r_lane = lane % RD, h_lane = lane / RD;
  const float eta_r = K.eta_r, sr = K.shift_r[r_lane];
  int na = 0;

  // ---- radial terms + angular neighbour staging --------------------------------
  for (int k0 = 0; k0 < cnt; k0 += 32) {
    int k = k0 + lane;
    float d = 0.f, fc = 0.f;
    int sj = -1;
    bool is_ang = false;
    float vx = 0.f, vy = 0.f, vz = 0.f;
    if (k < cnt) {
      int j = __ldg(nbr_j + row + k);
      unsigned sh = __ldg(nbr_shift + row + k);
      float4 pj = xyzs[j];
      edge_vec(pi, pj, sh, c, vx, vy, vz);
      float d2 = dist2_exact(vx, vy, vz);
      d = sqrtf(fmaxf(d2, 1e-5f));
      fc = d < K.rc ? 0.5f * cosf(d * K.pi_rc) + 0.5f : 0.f;
      sj = __float_as_int(pj.w);
      is_ang = d2 < K.rca2;
    }
    // stage radial data (d, 0.25*fc, species) in the triplet staging area
    sm.stA[lane] = d;
    sm.stA[32 + lane] = 0.25f * fc;
    ((int*)sm.stB)[lane] = sj;
    unsigned m = __ballot_sync(0xffffffffu, is_ang);
    if (is_ang) {
      int pos = na + warp_exclusive_prefix(m, lane);
      if (pos < kCapA) {
        float inv = 1.0f / fmaxf(d, 1e-5f);
        sm.au[4 * pos + 0] = vx * inv;
        sm.au[4 * pos + 1] = vy * inv;
        sm.au[4 * pos + 2] = vz * inv;
        sm.au[4 * pos + 3] = d;
        sm.afc[pos] = d < K.rca ? 0.5f * cosf(d * K.pi_rca) + 0.5f : 0.f;
        sm.asp[pos] = sj;
      }
    }
    na += __popc(m);
    __syncwarp();
    int nt = min(32, cnt - k0);
    for (int t = h_lane; t < nt; t += nh) {
      int s = ((int*)sm.stB)[t];
      float dd = sm.stA[t] - sr;
      float v = sm.stA[32 + t] * expf(-eta_r * dd * dd);
      sm.rad[s * 32 + lane] += v;
    }
    __syncwarp();
  }
  if (lane == 0) {
    status_max(status, ST_ANG_MAXCOUNT, na);
    if (na > kCapA) status_set(status, ST_ANG_OVERFLOW);
  }
  if (na > kCapA) na = kCapA;

  // ---- angular terms over all unordered neighbour pairs -----------------------
  const int T = na * (na - 1) / 2;
  const int fr = lane / AS, fz = lane % AS;  // feature (r, z) of this lane
  for (int t0 = 0; t0 < T; t0 += 32) {
    int t = t0 + lane;
    int p = -1;
    if (t < T) {
      int a, b;
      triplet_ab(t, a, b);
      float ax = sm.au[4 * a], ay = sm.au[4 * a + 1], az = sm.au[4 * a + 2], da = sm.au[4 * a + 3];
      float bx = sm.au[4 * b], by = sm.au[4 * b + 1], bz = sm.au[4 * b + 2], db = sm.au[4 * b + 3];
      float cosang = ax * bx + ay * by + az * bz;
      float ct = 0.95f * cosang;
      float st = sqrtf(fmaxf(1.0f - ct * ct, 0.f));
      float f = K.c_ang * sm.afc[a] * sm.afc[b];
#pragma unroll
      for (int z = 0; z < AS; ++z) {
        float cz = ct * K.cosz[z] + st * K.sinz[z];
        sm.stA[lane * 33 + z] = f * powf(fmaxf(1.0f + cz, 0.f), K.zeta);
      }
      float dm = 0.5f * (da + db);
#pragma unroll
      for (int r = 0; r < AD; ++r) {
        float x = dm - K.shift_a[r];
        sm.stB[lane * 33 + r] = expf(-K.eta_a * x * x);
      }
      p = triu_pair(sm.asp[a], sm.asp[b], S);
    }
    sm.stP[lane] = p;
    __syncwarp();
    int nt = min(32, T - t0);
    float* acc_col = sm.ang + lane;
    for (int tt = 0; tt < nt; ++tt) {
      int pp = sm.stP[tt];
      acc_col[pp * 32] += sm.stA[tt * 33 + fz] * sm.stB[tt * 33 + fr];
    }
    __syncwarp();
  }

  // ---- write the AEV row ------------------------------------------------------
  const size_t orow = (size_t)atom_row[i] * ld;
  const int F = K.F, FR = S * RD;
  for (int col = lane; col < F; col += 32) {
    float v;
    if (col < FR) {
      int s = col / RD, r = col % RD;
      v = 0.f;
      for (int h = 0; h < nh; ++h) v += sm.rad[s * 32 + r + RD * h];
    } else {
      v = sm.ang[col - FR];
    }
    if (out_kind == FENNOL_AEV_F32) {
      ((float*)out)[orow + col] = v;
    } else {
      __nv_bfloat16 hi = to_bf16(v);
      ((__nv_bfloat16*)out)[orow + col] = hi;
      if (out_kind == FENNOL_AEV_BF16X2)
        ((__nv_bfloat16*)out_lo)[orow + col] = to_bf16(v - __bfloat162float(hi));
    }
  }
}

// --------------------------------------------------------------------------------
// Adjoint: dE/dAEV -> forces.
// --------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int bwd_smem_floats(int S, int P, int cap) {
  return S * 33 + P * 33 + kCapA * 8 + cap * 4;
}

template <int RD, int AD, int AS>
__global__ void __launch_bounds__(kAevWarps * 32)
k_aev_backward(const float4* __restrict__ xyzs, int n, const int* __restrict__ atom_sys,
               const float* __restrict__ sys_cell, const int* __restrict__ nbr_j,
               const unsigned* __restrict__ nbr_shift, const int* __restrict__ nbr_count, int cap,
               const AevConst K, const int* __restrict__ atom_row, const float* __restrict__ daev,
               int ld, float4* __restrict__ forces, int* status) {
  extern __shared__ float smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kAevWarps + warp;
  if (i >= n) return;
  const int S = K.S, P = K.P;
  float* gr = smem + (size_t)warp * bwd_smem_floats(S, P, cap);  // [S][33]
  float* ga = gr + S * 33;                                         // [P][33]
  float* au = ga + P * 33;                                         // [kCapA][4]
  float* afc = au + kCapA * 4;                                     // [kCapA]
  float* adfc = afc + kCapA;                                       // [kCapA]
  int* asp = (int*)(adfc + kCapA);                                 // [kCapA]
  int* aslot = asp + kCapA;                                        // [kCapA]
  float* grad = (float*)(aslot + kCapA);                           // [cap][4]

  // dE/dAEV row -> shared memory (padded rows avoid bank conflicts)
  const float* g = daev + (size_t)atom_row[i] * ld;
  const int FR = S * RD;
  for (int col = lane; col < FR; col += 32) gr[(col / RD) * 33 + col % RD] = g[col];
  for (int col = lane; col < P * 32; col += 32) ga[(col >> 5) * 33 + (col & 31)] = g[FR + col];

  const float4 pi = xyzs[i];
  float c[9];
  load_cell(sys_cell, atom_sys[i], c);
  int cnt = nbr_count[i];
  if (cnt > cap) cnt = cap;
  const size_t row = (size_t)i * cap;
  __syncwarp();

  // ---- radial: lane per neighbour --------------------------------------------
  int na = 0;
  for (int k0 = 0; k0 < cnt; k0 += 32) {
    int k = k0 + lane;
    bool is_ang = false;
    float vx = 0.f, vy = 0.f, vz = 0.f, d = 1.f, d2 = 0.f;
    int sj = 0;
    if (k < cnt) {
      int j = __ldg(nbr_j + row + k);
      unsigned sh = __ldg(nbr_shift + row + k);
      float4 pj = xyzs[j];
      edge_vec(pi, pj, sh, c, vx, vy, vz);
      d2 = dist2_exact(vx, vy, vz);
      d = sqrtf(fmaxf(d2, 1e-5f));
      sj = __float_as_int(pj.w);
      float fc = 0.f, dfc = 0.f;
      if (d < K.rc) {
        float sa, ca;
        sincosf(d * K.pi_rc, &sa, &ca);
        fc = 0.5f * ca + 0.5f;
        dfc = -0.5f * K.pi_rc * sa;
      }
      float dEdd = 0.f;
      const float* grow = gr + sj * 33;
#pragma unroll 8
      for (int r = 0; r < RD; ++r) {
        float x = d - K.shift_r[r];
        float e = expf(-K.eta_r * x * x);
        dEdd += grow[r] * e * (dfc - 2.f * K.eta_r * x * fc);
      }
      dEdd *= 0.25f;
      float s = d2 > 1e-5f ? dEdd / d : 0.f;
      grad[4 * k + 0] = s * vx;
      grad[4 * k + 1] = s * vy;
      grad[4 * k + 2] = s * vz;
      is_ang = d2 < K.rca2;
    }
    unsigned m = __ballot_sync(0xffffffffu, is_ang);
    if (is_ang) {
      int pos = na + warp_exclusive_prefix(m, lane);
      if (pos < kCapA) {
        float inv = 1.0f / fmaxf(d, 1e-5f);
        au[4 * pos + 0] = vx * inv;
        au[4 * pos + 1] = vy * inv;
        au[4 * pos + 2] = vz * inv;
        au[4 * pos + 3] = d;
        float fc = 0.f, dfc = 0.f;
        if (d < K.rca) {
          float sa, ca;
          sincosf(d * K.pi_rca, &sa, &ca);
          fc = 0.5f * ca + 0.5f;
          dfc = -0.5f * K.pi_rca * sa;
        }
        afc[pos] = fc;
        adfc[pos] = dfc;
        asp[pos] = sj;
        aslot[pos] = k;
      }
    }
    na += __popc(m);
  }
  if (na > kCapA) {
    if (lane == 0) status_set(status, ST_ANG_OVERFLOW);
    na = kCapA;
  }
  __syncwarp();

  // ---- angular: lane per triplet -----------------------------------------------
  const int T = na * (na - 1) / 2;
  const float zeta = K.zeta;
  for (int t = lane; t < T; t += 32) {
    int a, b;
    triplet_ab(t, a, b);
    float uax = au[4 * a], uay = au[4 * a + 1], uaz = au[4 * a + 2], da = au[4 * a + 3];
    float ubx = au[4 * b], uby = au[4 * b + 1], ubz = au[4 * b + 2], db = au[4 * b + 3];
    float cosang = uax * ubx + uay * uby + uaz * ubz;
    float ct = 0.95f * cosang;
    float st = sqrtf(fmaxf(1.0f - ct * ct, 1e-12f));
    int p = triu_pair(asp[a], asp[b], S);
    const float* gp = ga + p * 33;
    float A[AS], Ap[AS];
#pragma unroll
    for (int z = 0; z < AS; ++z) {
      float cz = ct * K.cosz[z] + st * K.sinz[z];
      float sz = st * K.cosz[z] - ct * K.sinz[z];  // sin(theta - Z)
      float base = fmaxf(1.0f + cz, 0.f);
      float pw1 = base > 0.f ? powf(base, zeta - 1.0f) : 0.f;
      A[z] = pw1 * base;
      Ap[z] = -zeta * pw1 * sz;
    }
    float dm = 0.5f * (da + db);
    float Q = 0.f, Th = 0.f, Dm = 0.f;
#pragma unroll
    for (int r = 0; r < AD; ++r) {
      float x = dm - K.shift_a[r];
      float B = expf(-K.eta_a * x * x);
      float GA = 0.f, GAp = 0.f;
#pragma unroll
      for (int z = 0; z < AS; ++z) {
        float gv = gp[r * AS + z];
        GA += gv * A[z];
        GAp += gv * Ap[z];
      }
      Q += GA * B;
      Th += GAp * B;
      Dm += GA * (-2.f * K.eta_a * x * B);
    }
    float fa = afc[a], fb = afc[b];
    float C = K.c_ang;
    float dEdth = C * fa * fb * Th;
    float dEddm = C * fa * fb * Dm;
    float dEdda = 0.5f * dEddm + C * fb * Q * adfc[a];
    float dEddb = 0.5f * dEddm + C * fa * Q * adfc[b];
    float dEdc = dEdth * (-0.95f / st);
    float ia = dEdc / da, ib = dEdc / db;
    float gax = dEdda * uax + ia * (ubx - cosang * uax);
    float gay = dEdda * uay + ia * (uby - cosang * uay);
    float gaz = dEdda * uaz + ia * (ubz - cosang * uaz);
    float gbx = dEddb * ubx + ib * (uax - cosang * ubx);
    float gby = dEddb * uby + ib * (uay - cosang * uby);
    float gbz = dEddb * ubz + ib * (uaz - cosang * ubz);
    int sa_ = aslot[a], sb_ = aslot[b];
    atomicAdd(grad + 4 * sa_ + 0, gax);
    atomicAdd(grad + 4 * sa_ + 1, gay);
    atomicAdd(grad + 4 * sa_ + 2, gaz);
    atomicAdd(grad + 4 * sb_ + 0, gbx);
    atomicAdd(grad + 4 * sb_ + 1, gby);
    atomicAdd(grad + 4 * sb_ + 2, gbz);
  }
  __syncwarp();

  // ---- scatter: F_j -= g, F_i += sum g ----------------------------------------
  float fx = 0.f, fy = 0.f, fz = 0.f;
  for (int k = lane; k < cnt; k += 32) {
    float gx = grad[4 * k], gy = grad[4 * k + 1], gz = grad[4 * k + 2];
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
}

__global__ void k_pack(const float* __restrict__ coords, const int* __restrict__ sp, int n,
                       float4* __restrict__ xyzs) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  xyzs[i] = make_float4(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], __int_as_float(sp[i]));
}

template <int RD, int AD, int AS>
struct AevKernels {
  static constexpr auto fwd = k_aev_forward<RD, AD, AS>;
  static constexpr auto bwd = k_aev_backward<RD, AD, AS>;
};

// (RD, AD, AS) combinations compiled: radial 16/32 x angular (8,4) / (4,8).
template <typename Fn>
bool dispatch(const AevConst& K, Fn&& fn) {
  if (K.RD == 16 && K.AD == 8 && K.AS == 4) return fn(AevKernels<16, 8, 4>{});
  if (K.RD == 16 && K.AD == 4 && K.AS == 8) return fn(AevKernels<16, 4, 8>{});
  if (K.RD == 32 && K.AD == 8 && K.AS == 4) return fn(AevKernels<32, 8, 4>{});
  if (K.RD == 32 && K.AD == 4 && K.AS == 8) return fn(AevKernels<32, 4, 8>{});
  return false;
}

size_t set_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) {
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
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

extern "C" int fennol_pack_atoms(const float* coords, const int* species_idx, int natoms, float* xyzs,
                                 void* stream) {
  if (natoms < 0 || (natoms > 0 && (!coords || !species_idx || !xyzs))) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  k_pack<<<(natoms + 255) / 256, 256, 0, (cudaStream_t)stream>>>(coords, species_idx, natoms,
                                                                  (float4*)xyzs);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_aev_forward(const float* xyzs, int natoms, const int* atom_sys,
                                  const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                                  const int* nbr_count, int capacity, const fennol_aev_params* p,
                                  const int* atom_row, int out_kind, void* out, void* out_lo, int ld,
                                  int* status, void* stream) {
  AevConst K;
  if (!make_const(p, &K)) return FENNOL_ERR_UNSUPPORTED;
  if (natoms < 0 || capacity <= 0 || ld < K.F) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!xyzs || !atom_sys || !nbr_j || !nbr_shift || !nbr_count || !atom_row || !out)
    return FENNOL_ERR_INVALID;
  if (out_kind != FENNOL_AEV_F32 && out_kind != FENNOL_AEV_BF16 && out_kind != FENNOL_AEV_BF16X2)
    return FENNOL_ERR_INVALID;
  if (out_kind == FENNOL_AEV_BF16X2 && !out_lo) return FENNOL_ERR_INVALID;
  int blocks = (natoms + kAevWarps - 1) / kAevWarps;
  bool launched = dispatch(K, [&](auto ks) {
    size_t smem = set_smem((const void*)ks.fwd,
                           (size_t)kAevWarps * fwd_smem_floats(K.S, K.P) * sizeof(float));
    if (!smem) return false;
    ks.fwd<<<blocks, kAevWarps * 32, smem, (cudaStream_t)stream>>>(
        (const float4*)xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, K,
        atom_row, out_kind, out, out_lo, ld, status);
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
  AevConst K;
  if (!make_const(p, &K)) return FENNOL_ERR_UNSUPPORTED;
  if (natoms < 0 || capacity <= 0 || ld < K.F) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!xyzs || !atom_sys || !nbr_j || !nbr_shift || !nbr_count || !atom_row || !daev || !forces4)
    return FENNOL_ERR_INVALID;
  size_t bytes = (size_t)kAevWarps * bwd_smem_floats(K.S, K.P, capacity) * sizeof(float);
  if (bytes > 200 * 1024) return FENNOL_ERR_UNSUPPORTED;
  int blocks = (natoms + kAevWarps - 1) / kAevWarps;
  bool launched = dispatch(K, [&](auto ks) {
    size_t smem = set_smem((const void*)ks.bwd, bytes);
    if (!smem) return false;
    ks.bwd<<<blocks, kAevWarps * 32, smem, (cudaStream_t)stream>>>(
        (const float4*)xyzs, natoms, atom_sys, sys_cell, nbr_j, nbr_shift, nbr_count, capacity, K,
        atom_row, daev, ld, (float4*)forces4, status);
    return true;
  });
  if (!launched) return FENNOL_ERR_UNSUPPORTED;
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}
