// Fused, persistent species MLP on tcgen05 (sm_100a): forward + input gradient
// of FullyConnectedNet (src/fennol/models/misc/nets.py:13-102) inside
// SpeciesIndexNet (:301-426), with the ensemble mean, in one launch.
//
// One CTA per SM loops over 128-row tiles (one species each) and, for every
// model of the ensemble, runs the six GEMMs of the layer chain
//     L1 X.W1  L2 H1.W2  L3 H2.W3 (+ energy head)  B3 G3.W3^T  B2 G2.W2^T  B1 G1.W1^T
// keeping the activations on chip:
//   * warp 0 (one thread) streams the AEV tile and W1^T through a 3-stage TMA
//     ring (2 stages when the W1^T low parts come along) that aliases the
//     activation buffer and the weight ring, then all other weights through
//     the 2-stage weight ring;
//   * warp 1 owns the 512 TMEM columns (two 256-column FP32 accumulators used
//     alternately) and one thread issues tcgen05.mma / tcgen05.commit;
//   * warps 2-9 are the epilogue: they read an accumulator (tcgen05.ld, one
//     row per thread, two warps per lane quarter), apply bias + CELU, the energy
//     head, or CELU' masks, and write the next A operand as 16-bit hi (+ lo)
//     pairs straight into shared memory in the 128-byte-swizzled K-major
//     layout the MMA descriptors expect (fence.proxy.async before the MMA
//     reads it).
// Operand forms: BF16 (A hi, optionally A lo; weights BF16) and FP16 (the
// kernel template's F16 flag).  The FP16 forms split the activations and the
// power-of-two-scaled float32 weights into float16 hi + lo: the forward GEMMs
// run A_hi W_hi + A_lo W_hi + A_hi W_lo, the input-gradient GEMMs G_hi W_hi
// (+ G_hi W_lo).  Each epilogue divides its accumulator by the layer's weight
// scale; the backward chain carries the power-of-two scale of the last layer's
// kernel until dX.
// Active columns: bit c of kmask says that input columns [64c, 64c + 64) may
// be non-zero (the caller guarantees the others are zero in every row).  L1
// streams only the active K-chunks, and B1 computes dX only on runs of up to
// four consecutive active chunks (the other dX columns are left untouched).
// CELU' of layers 1-2 (needed by the backward) goes to a per-CTA scratch in
// global memory that stays L2 resident.  The ensemble is processed model by
// model inside the CTA, so the per-row energy and dE/dAEV sums are
// deterministic.  Every wait is bounded (2 s); a timeout sets the error word,
// raises a shared abort flag that ends all roles, and the CTA frees its TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "mlp_common.cuh"
#include "umma.cuh"

using namespace fnl;
using namespace fnl::umma;

namespace {

constexpr int kThreads = 320;
constexpr int kEpiThreads = 256;
constexpr int BM = 128, BK = 64;
constexpr uint32_t kAtom = BM * BK * 2;           // one 128 x 64 BF16 K-atom: 16 KB
constexpr uint32_t kActHalf = 4 * kAtom;          // up to K = 256 per hi (or lo) operand
constexpr uint32_t kActBytes = 2 * kActHalf;      // 128 KB
constexpr int kWStages = 2;
constexpr uint32_t kWStage = 256 * BK * 2;        // 32 KB
constexpr uint32_t kXStage = kActBytes / 2;       // 64 KB: A hi | A lo | B (<= 256 rows)
// L1 ring: stages 0-1 alias the activation buffer, stage 2 the weight ring
// (idle while L1 streams); stage s starts at act + s * kXStage.  With the W1^T
// low parts a stage is A hi | A lo | B hi | B lo (96 KB) and the ring has two
// stages, the second one aliasing the weight ring.
constexpr int kXStages = 3;
constexpr uint32_t kXStageWide = 6 * kAtom;       // 96 KB
constexpr int kXStagesWide = 2;
constexpr uint32_t kXpose = 8 * 32 * 32 * 4;      // per-epilogue-warp 32x32 dX staging tiles: 32 KB
constexpr uint32_t kSmemMain = kActBytes + kWStages * kWStage + kXpose;  // 224 KB
// bounded waits: default limit, and the settings of fennol_mlp_wait_limit /
// fennol_mlp_inject_stall (host side)
constexpr uint64_t kTimeoutNs = 2000000000ull;
uint64_t g_wait_limit_ns = kTimeoutNs;
int g_stall_launches = 0;

struct FusedParams {
  int ntiles, n_models, n_species;
  const int* tile_species;
  const int* tile_row;
  int d0, d1, d2, d3;
  int a_lo;   // forward A operands (X, H1, H2) carry a lo part
  int g_lo;   // input-gradient A operands (G3, G2, G1) carry a lo part
  int wf_lo;  // forward GEMMs add A_hi x W_lo
  int wb_lo;  // input-gradient GEMMs add G_hi x W_lo
  int xstages;
  uint32_t xstage;
  float alpha, inv_models;
  unsigned long long kmask;  // active 64-column chunks of the input
  unsigned long long timeout_ns;  // limit of every bounded wait
  int stall;                      // the load producer issues no copies (timeout tests)
  const float4* scales;  // F16 forms: per group (s_W1, s_W2, s_W3, s_w4) powers of two
  const float* b1;
  const float* b2;
  const float* b3;
  const float* w4;
  const float* b4;
  float* e_rows;
  float* dx;
  float* dc;  // [gridDim.x][128][d1 + d2]
  int* err;
};

struct Maps {
  CUtensorMap x, xlo, w1t, w2t, w3t, w3, w2, w1;
  CUtensorMap w1t_lo, w2t_lo, w3t_lo, w3_lo, w2_lo, w1_lo;  // low parts (unused maps alias the high ones)
  CUtensorMap dx;  // FP32 [rows][d0], 32 x 32 boxes, 128-byte swizzle
};

struct Bars {
  uint64_t x_full[kXStages], x_empty[kXStages], w_full[kWStages], w_empty[kWStages];
  uint64_t acc_full[2], acc_free[2], act_ready[4], act_free, done, ex_ready, ex_free;
  uint32_t tmem_slot;
  int abort_flag;
  float ex[BM];
};

// First active 64-column chunk at or after c and the length (at most 4) of
// the run of consecutive active chunks that starts there; -1 when none is left.
__device__ __forceinline__ int run_at(unsigned long long mask, int c, int& len) {
  const unsigned long long m = c < 64 ? (mask >> c) : 0ull;
  if (!m) {
    len = 0;
    return -1;
  }
  const int s = c + __ffsll((long long)m) - 1;
  int l = 1;
  while (l < 4 && s + l < 64 && ((mask >> (s + l)) & 1ull)) ++l;
  len = l;
  return s;
}

// Drop the 128-byte L2 line at a (128-byte aligned) without writing it back;
// its contents become undefined.
__device__ __forceinline__ void discard_l2(const void* a) {
  asm volatile("discard.global.L2 [%0], 128;" ::"l"(a) : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// CELU and its derivative from one exponential: e = exp(z/alpha) for z <= 0,
// celu = alpha (e - 1), celu' = e; both are z and 1 for z > 0.
__device__ __forceinline__ void celu_pair(float z, float alpha, float k2, float& h, float& dh) {
  // k2 = log2(e) / alpha: e = 2^(min(z, 0) k2) by the SFU
  float e;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(fminf(z, 0.f) * k2));
  h = z > 0.f ? z : fmaf(alpha, e, -alpha);
  dh = z > 0.f ? 1.f : e;
}

// Bounded wait that also gives up when another role has aborted.
// Threads sleep in mbarrier.try_wait (woken when the phase completes) instead
// of polling, so waiting epilogue warps do not take issue slots from the MMA
// and TMA threads.
__device__ __forceinline__ bool wait_bar(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                         uint64_t p_timeout_ns) {
  if (mbar_try(bar, parity, 20000u)) return true;
  const uint64_t deadline = globaltimer() + p_timeout_ns;
  while (true) {
    if (mbar_try(bar, parity, 20000u)) return true;
    if (*abort_flag) return false;
    if (globaltimer() > deadline) {
      *abort_flag = 1;
      atomicExch(err, 1);
      return false;
    }
  }
}

// Write 32 consecutive columns [n, n+32) of row r as 16-bit hi (+ lo) into the
// swizzled K-major activation buffer (BF16, or FP16 when F16).
template <bool F16>
__device__ __forceinline__ void act_store(uint8_t* act, int r, int n, const float* v, bool with_lo) {
  uint32_t h[16], l[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    // one paired conversion per two columns for the high parts and one for the
    // residuals (round to nearest each, as two single conversions would)
    if constexpr (F16) {
      const __half2 hb = __floats2half2_rn(v[2 * k], v[2 * k + 1]);
      const float2 hf = __half22float2(hb);
      const __half2 lb = __floats2half2_rn(v[2 * k] - hf.x, v[2 * k + 1] - hf.y);
      h[k] = *reinterpret_cast<const uint32_t*>(&hb);
      l[k] = *reinterpret_cast<const uint32_t*>(&lb);
    } else {
      const __nv_bfloat162 hb = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
      const float2 hf = __bfloat1622float2(hb);
      const __nv_bfloat162 lb = __floats2bfloat162_rn(v[2 * k] - hf.x, v[2 * k + 1] - hf.y);
      h[k] = *reinterpret_cast<const uint32_t*>(&hb);
      l[k] = *reinterpret_cast<const uint32_t*>(&lb);
    }
  }
  const int atom = n >> 6;
  const int j0 = (n & 63) >> 3;
  const uint32_t rowoff = (uint32_t)(r >> 3) * 1024u + (uint32_t)(r & 7) * 128u;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint32_t off = rowoff + (uint32_t)(((j0 + q) ^ (r & 7)) << 4);
    *reinterpret_cast<uint4*>(act + atom * kAtom + off) = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
    if (with_lo)
      *reinterpret_cast<uint4*>(act + kActHalf + atom * kAtom + off) =
          make_uint4(l[4 * q], l[4 * q + 1], l[4 * q + 2], l[4 * q + 3]);
  }
}

template <bool F16>
__global__ void __launch_bounds__(kThreads, 1) k_mlp_fused(const __grid_constant__ Maps maps, const FusedParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* act = smem;                     // 128 KB, aliased by the L1 ring
  uint8_t* wring = smem + kActBytes;       // 2 x 32 KB
  float* xpose = reinterpret_cast<float*>(smem + kActBytes + kWStages * kWStage);
  Bars* bars = reinterpret_cast<Bars*>(smem + kSmemMain);
  volatile int* abort_flag = &bars->abort_flag;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int M = p.n_models;
  const int XS = p.xstages;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kXStages; ++s) {
      mbar_init(&bars->x_full[s], 1);
      mbar_init(&bars->x_empty[s], 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(&bars->acc_full[s], 1);
      mbar_init(&bars->acc_free[s], kEpiThreads / 32);
    }
    for (int s = 0; s < kWStages; ++s) {
      mbar_init(&bars->w_full[s], 1);
      mbar_init(&bars->w_empty[s], 1);
    }
    for (int a = 0; a < 4; ++a) mbar_init(&bars->act_ready[a], kEpiThreads);
    mbar_init(&bars->act_free, 1);
    mbar_init(&bars->done, 1);
    mbar_init(&bars->ex_ready, kEpiThreads / 2);
    mbar_init(&bars->ex_free, kEpiThreads / 2);
    bars->abort_flag = 0;
    fence_barrier_init();
  }
  if (warp == 1) tmem_alloc(&bars->tmem_slot, 512);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = bars->tmem_slot;
  // Launched as a programmatic dependent of the AEV forward: the set-up above
  // (barriers, TMEM) touches no global memory and overlaps that kernel's last
  // wave; every role reads or writes global memory only after this wait.
  pdl_wait();

  const uint32_t x_tx = kAtom * (1 + p.a_lo) + (uint32_t)p.d1 * BK * 2 * (1 + p.wf_lo);

  if (warp == 0) {
    // ------------------------------------------------------------------ TMA producer
    // (with p.stall it issues nothing: the other roles' waits run out)
    if (lane == 0 && !p.stall) {
      const uint64_t keep = l2_evict_last();
      uint32_t xq = 0, wq = 0;
      int item = 0;
      bool ok = true;
      for (int w = blockIdx.x; w < p.ntiles && ok; w += gridDim.x) {
        const int row0 = p.tile_row[w];
        const int sp = p.tile_species[w];
        for (int m = 0; m < M && ok; ++m, ++item) {
          const int g = m * p.n_species + sp;
          if (item > 0 && !(ok = wait_bar(&bars->act_free, (item - 1) & 1, abort_flag, p.err, p.timeout_ns))) break;
          for (unsigned long long rest = p.kmask; rest; rest &= rest - 1, ++xq) {
            const int kc = __ffsll((long long)rest) - 1;
            const int s = xq % XS;
            const uint32_t u = xq / XS;
            if (u > 0 && !(ok = wait_bar(&bars->x_empty[s], (u - 1) & 1, abort_flag, p.err, p.timeout_ns))) break;
            uint8_t* st = act + s * p.xstage;
            mbar_expect_tx(&bars->x_full[s], x_tx);
            // the AEV tile is read once per model: kept in L2 ahead of other lines
            tma_load_2d_hint(&maps.x, &bars->x_full[s], st, kc * BK, row0, keep);
            if (p.a_lo) tma_load_2d_hint(&maps.xlo, &bars->x_full[s], st + kAtom, kc * BK, row0, keep);
            tma_load_2d(&maps.w1t, &bars->x_full[s], st + 2 * kAtom, kc * BK, g * p.d1);
            if (p.wf_lo) tma_load_2d(&maps.w1t_lo, &bars->x_full[s], st + 4 * kAtom, kc * BK, g * p.d1);
          }
          if (!ok) break;
          // the weight ring lies in the last L1 stage: its latest chunk must have
          // been consumed (a stage last used by an earlier item was, before
          // act_free completed)
          {
            const int rs = XS - 1;
            if (xq > (uint32_t)rs) {
              const uint32_t last = xq - 1 - ((xq - 1 - rs) % XS);
              if (!(ok = wait_bar(&bars->x_empty[rs], (last / XS) & 1, abort_flag, p.err, p.timeout_ns))) break;
            }
          }
          // weight chunks of the remaining GEMMs, in MMA order
          // (a GEMM with weight low parts takes the hi and lo chunks of each K step)
          const CUtensorMap* wm[4] = {&maps.w2t, &maps.w3t, &maps.w3, &maps.w2};
          const CUtensorMap* wml[4] = {&maps.w2t_lo, &maps.w3t_lo, &maps.w3_lo, &maps.w2_lo};
          const int rows_g[4] = {p.d2, p.d3, p.d2, p.d1};
          const int nk[4] = {p.d1 / BK, p.d2 / BK, p.d3 / BK, p.d2 / BK};
          const int nt[4] = {1 + p.wf_lo, 1 + p.wf_lo, 1 + p.wb_lo, 1 + p.wb_lo};
          for (int jb = 0; jb < 4 && ok; ++jb) {
            for (int kc = 0; kc < nk[jb] && ok; ++kc) {
              for (int t = 0; t < nt[jb]; ++t, ++wq) {
                const int s = wq % kWStages;
                const uint32_t u = wq / kWStages;
                if (u > 0 && !(ok = wait_bar(&bars->w_empty[s], (u - 1) & 1, abort_flag, p.err, p.timeout_ns))) break;
                mbar_expect_tx(&bars->w_full[s], (uint32_t)rows_g[jb] * BK * 2);
                tma_load_2d(t ? wml[jb] : wm[jb], &bars->w_full[s], wring + s * kWStage, kc * BK, g * rows_g[jb]);
              }
            }
          }
          // B1: W1 rows of each run of active dX chunks, 64-row boxes stacked in the stage
          for (int len = 0, c0 = run_at(p.kmask, 0, len); c0 >= 0 && ok; c0 = run_at(p.kmask, c0 + len, len)) {
            for (int kc = 0; kc < p.d1 / BK && ok; ++kc) {
              for (int t = 0; t < 1 + p.wb_lo; ++t, ++wq) {
                const int s = wq % kWStages;
                const uint32_t u = wq / kWStages;
                if (u > 0 && !(ok = wait_bar(&bars->w_empty[s], (u - 1) & 1, abort_flag, p.err, p.timeout_ns))) break;
                mbar_expect_tx(&bars->w_full[s], (uint32_t)len * 64 * BK * 2);
                for (int q = 0; q < len; ++q)
                  tma_load_2d(t ? &maps.w1_lo : &maps.w1, &bars->w_full[s], wring + s * kWStage + q * 64 * BK * 2,
                              kc * BK, g * p.d0 + (c0 + q) * 64);
              }
            }
          }
        }
      }
      // Before the CTA can exit, every issued TMA load must have landed (on an
      // abort some stages may never be consumed).  Bounded, ignores the abort flag.
      int dummy = 0;
      for (uint32_t s = 0; s < (uint32_t)XS && s < xq; ++s) {
        const uint32_t last = xq - 1 - ((xq - 1 - s) % XS);
        wait_bar(&bars->x_full[s], (last / XS) & 1, &dummy, p.err, p.timeout_ns);
      }
      for (uint32_t s = 0; s < (uint32_t)kWStages && s < wq; ++s) {
        const uint32_t last = wq - 1 - ((wq - 1 - s) % kWStages);
        wait_bar(&bars->w_full[s], (last / kWStages) & 1, &dummy, p.err, p.timeout_ns);
      }
    }
  } else if (warp == 1) {
    // ------------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      uint32_t xq = 0, wq = 0;
      uint32_t act_phase[4] = {0, 0, 0, 0};
      uint32_t nuse[2] = {0, 0};
      uint32_t job = 0;
      bool ok = true;
      const uint32_t act_hi = smem_u32(act), act_lo = smem_u32(act + kActHalf);
      auto acquire_acc = [&](uint32_t b) -> bool {
        if (nuse[b] == 0) return true;
        return wait_bar(&bars->acc_free[b], (nuse[b] - 1) & 1, abort_flag, p.err, p.timeout_ns);
      };
      // one GEMM whose A operand is the activation buffer (K/64 atoms) and B the
      // weight ring.  With wait_act, each K-atom is used as soon as the epilogue
      // has published it, so the GEMM overlaps the epilogue that feeds it.
      // alo: A carries a lo part; wlo: each K step also has a W lo chunk.
      auto gemm_act = [&](int n, int k, uint32_t b, bool wait_act, bool alo, bool wlo) -> bool {
        const uint32_t idesc = F16 ? idesc_f16_f32(n) : idesc_bf16_f32(n);
        const uint32_t d = tmem + b * 256;
        for (int kc = 0; kc < k / BK; ++kc) {
          if (wait_act) {
            if (!wait_bar(&bars->act_ready[kc], act_phase[kc] & 1, abort_flag, p.err, p.timeout_ns)) return false;
            ++act_phase[kc];
          }
          int s = wq % kWStages;
          if (!wait_bar(&bars->w_full[s], (wq / kWStages) & 1, abort_flag, p.err, p.timeout_ns)) return false;
          fence_after_sync();
          uint32_t bs = smem_u32(wring + s * kWStage);
#pragma unroll
          for (int kk = 0; kk < BK / 16; ++kk) {
            const uint64_t bd = sdesc_sw128(bs + kk * 32);
            mma_bf16(d, sdesc_sw128(act_hi + kc * kAtom + kk * 32), bd, idesc, (kc | kk) != 0);
            if (alo) mma_bf16(d, sdesc_sw128(act_lo + kc * kAtom + kk * 32), bd, idesc, 1u);
          }
          mma_commit(&bars->w_empty[s]);
          ++wq;
          if (wlo) {
            s = wq % kWStages;
            if (!wait_bar(&bars->w_full[s], (wq / kWStages) & 1, abort_flag, p.err, p.timeout_ns)) return false;
            fence_after_sync();
            bs = smem_u32(wring + s * kWStage);
#pragma unroll
            for (int kk = 0; kk < BK / 16; ++kk)
              mma_bf16(d, sdesc_sw128(act_hi + kc * kAtom + kk * 32), sdesc_sw128(bs + kk * 32), idesc, 1u);
            mma_commit(&bars->w_empty[s]);
            ++wq;
          }
        }
        return true;
      };
      for (int w = blockIdx.x; w < p.ntiles && ok; w += gridDim.x) {
        for (int m = 0; m < M && ok; ++m) {
          // L1: A and B from the X ring
          {
            const uint32_t b = job & 1;
            if (!(ok = acquire_acc(b))) break;
            const uint32_t idesc = F16 ? idesc_f16_f32(p.d1) : idesc_bf16_f32(p.d1);
            const uint32_t d = tmem + b * 256;
            int ki = 0;
            for (unsigned long long rest = p.kmask; rest; rest &= rest - 1, ++xq, ++ki) {
              const int s = xq % XS;
              if (!(ok = wait_bar(&bars->x_full[s], (xq / XS) & 1, abort_flag, p.err, p.timeout_ns))) break;
              fence_after_sync();
              const uint32_t st = smem_u32(act + s * p.xstage);
#pragma unroll
              for (int kk = 0; kk < BK / 16; ++kk) {
                const uint64_t ad = sdesc_sw128(st + kk * 32);
                const uint64_t bd = sdesc_sw128(st + 2 * kAtom + kk * 32);
                mma_bf16(d, ad, bd, idesc, (ki | kk) != 0);
                if (p.a_lo) mma_bf16(d, sdesc_sw128(st + kAtom + kk * 32), bd, idesc, 1u);
                if (p.wf_lo) mma_bf16(d, ad, sdesc_sw128(st + 4 * kAtom + kk * 32), idesc, 1u);
              }
              mma_commit(&bars->x_empty[s]);
            }
            if (!ok) break;
            mma_commit(&bars->acc_full[b]);
            ++nuse[b];
            ++job;
          }
          // L2, L3, B3, B2: A from the activation buffer written by the epilogue
          const int ns[4] = {p.d2, p.d3, p.d2, p.d1};
          const int ks[4] = {p.d1, p.d2, p.d3, p.d2};
          for (int jb = 0; jb < 4 && ok; ++jb) {
            const uint32_t b = job & 1;
            const bool fwd = jb < 2;
            if (!(ok = acquire_acc(b))) break;
            if (!(ok = gemm_act(ns[jb], ks[jb], b, true, fwd ? p.a_lo : p.g_lo, fwd ? p.wf_lo : p.wb_lo))) break;
            mma_commit(&bars->acc_full[b]);
            ++nuse[b];
            ++job;
          }
          if (!ok) break;
          // B1: dX on each run of active chunks (<= 256 columns), A = G1
          // (published atom by atom for the first run)
          bool first = true;
          for (int len = 0, c0 = run_at(p.kmask, 0, len); c0 >= 0 && ok; c0 = run_at(p.kmask, c0 + len, len)) {
            const uint32_t b = job & 1;
            if (!(ok = acquire_acc(b))) break;
            if (!(ok = gemm_act(64 * len, p.d1, b, first, p.g_lo, p.wb_lo))) break;
            first = false;
            mma_commit(&bars->acc_full[b]);
            ++nuse[b];
            ++job;
          }
          if (!ok) break;
          mma_commit(&bars->act_free);
        }
      }
      // all issued MMAs complete before TMEM is released
      mma_commit(&bars->done);
      wait_bar(&bars->done, 0, abort_flag, p.err, p.timeout_ns);
    }
  } else {
    // ------------------------------------------------------------------ epilogue
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int r = 32 * q + lane;
    const uint32_t lane_base = (uint32_t)(32 * q) << 16;
    uint32_t nuse[2] = {0, 0};
    uint32_t job = 0, ex_phase = 0;
    bool ok = true;
    // per-CTA CELU' scratch, column-major [d1 + d2][128] so that a warp's 32 rows are contiguous
    float* dc = p.dc + (size_t)blockIdx.x * BM * (p.d1 + p.d2) + r;
    // this warp's 128-byte segment (32 rows) of CELU' column 0
    float* dc_lines = p.dc + (size_t)blockIdx.x * BM * (p.d1 + p.d2) + 32 * q;
    const float celu_k2 = 1.4426950408889634f / p.alpha;  // log2(e) / alpha
    const bool with_lo = p.a_lo != 0;    // forward activations
    const bool grad_lo = p.g_lo != 0;    // input-gradient operands
    auto take_acc = [&](uint32_t b) -> bool {
      bool ready = __all_sync(0xffffffffu, wait_bar(&bars->acc_full[b], nuse[b] & 1, abort_flag, p.err, p.timeout_ns));
      if (ready) fence_after_sync();
      return ready;
    };
    auto release_acc = [&](uint32_t b) {
      fence_before_sync();
      __syncwarp();
      if (lane == 0) mbar_arrive(&bars->acc_free[b]);
      ++nuse[b];
      ++job;
    };
    // the 32 columns of K-atom a written by this thread are visible to the MMA
    // (async proxy); the atom is complete when all epilogue threads arrived
    auto publish_atom = [&](int a) {
      fence_proxy_async();
      mbar_arrive(&bars->act_ready[a]);
    };
    // H = celu(Z / s_W + bias) -> act for columns [0, n); celu'(z) / s_W' -> dc
    // columns [dc0, dc0 + n), where s_W' is the scale of the weights the
    // input gradient of this layer is taken through (a power of two, so the
    // product is exact).  The bias loads are issued before the TMEM load so
    // that their latencies overlap.  inv_s = 1 / s_W, dscale = 1 / s_W' (1 for
    // the BF16 forms).
    auto celu_layer = [&](uint32_t b, const float* bias, int n, int dc0, float inv_s, float dscale) {
      for (int cc = half; cc < n / 32; cc += 2) {
        float4 bb[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) bb[k] = __ldg(reinterpret_cast<const float4*>(bias + cc * 32) + k);
        float v[32];
        tmem_ld32(tmem + b * 256 + lane_base + cc * 32, v);
        float* dco = dc + (size_t)(dc0 + cc * 32) * BM;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float zz[4] = {fmaf(v[4 * k], inv_s, bb[k].x), fmaf(v[4 * k + 1], inv_s, bb[k].y),
                               fmaf(v[4 * k + 2], inv_s, bb[k].z), fmaf(v[4 * k + 3], inv_s, bb[k].w)};
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            float dh;
            celu_pair(zz[u], p.alpha, celu_k2, v[4 * k + u], dh);
            dco[(size_t)(4 * k + u) * BM] = dh * dscale;  // column-major: the warp writes 128 contiguous bytes
          }
        }
        act_store<F16>(act, r, cc * 32, v, with_lo);
        publish_atom(cc >> 1);
      }
    };
    // G = D / s_W * celu'(z) -> act for columns [0, n), celu'(z) / s_W read
    // back from dc columns [dc0, dc0 + n) (written by this thread); loads
    // issued before the TMEM load.
    auto mask_layer = [&](uint32_t b, int n, int dc0) {
      for (int cc = half; cc < n / 32; cc += 2) {
        const float* dci = dc + (size_t)(dc0 + cc * 32) * BM;
        float dd[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) dd[k] = dci[(size_t)k * BM];
        float v[32];
        tmem_ld32(tmem + b * 256 + lane_base + cc * 32, v);
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] *= dd[k];
        // the warp has read these 32 columns of its 32 rows for the last time:
        // their L2 lines are dropped without a write-back (the next item
        // rewrites them before reading)
        __syncwarp();
        discard_l2(dc_lines + (size_t)(dc0 + cc * 32 + lane) * BM);
        act_store<F16>(act, r, cc * 32, v, grad_lo);
        publish_atom(cc >> 1);
      }
    };
    for (int w = blockIdx.x; w < p.ntiles && ok; w += gridDim.x) {
      const int row = p.tile_row[w] + r;
      const int sp = p.tile_species[w];
      float e_row = 0.f;  // ensemble-mean row energy, accumulated model by model in registers
      for (int m = 0; m < M && ok; ++m) {
        const int g = m * p.n_species + sp;
        // weight scales of this group (powers of two: the reciprocals are exact)
        float inv_s1 = 1.f, inv_s2 = 1.f, inv_s3 = 1.f, s_g = 1.f;
        if constexpr (F16) {
          const float4 sc = __ldg(p.scales + g);
          inv_s1 = 1.f / sc.x;
          inv_s2 = 1.f / sc.y;
          inv_s3 = 1.f / sc.z;
          s_g = sc.w;
        }
        // E1: H1 = celu(Z1 + b1) -> act; celu'(z1) -> dc[0:d1]
        {
          const uint32_t b = job & 1;
          if (!(ok = take_acc(b))) break;
          celu_layer(b, p.b1 + (size_t)g * p.d1, p.d1, 0, inv_s1, inv_s2);
          release_acc(b);
        }
        // E2: H2 = celu(Z2 + b2) -> act; celu'(z2) -> dc[d1:d1+d2]
        {
          const uint32_t b = job & 1;
          if (!(ok = take_acc(b))) break;
          celu_layer(b, p.b2 + (size_t)g * p.d2, p.d2, p.d1, inv_s2, inv_s3);
          release_acc(b);
        }
        // E3: energy head; G3 = s_g w4 * celu'(z3) -> act.  Both column halves work;
        // the half-1 partial energy of each row reaches the half-0 thread through
        // shared memory guarded by two mbarriers (bounded waits, no CTA barrier).
        {
          const uint32_t b = job & 1;
          if (!(ok = take_acc(b))) break;
          const float* bias = p.b3 + (size_t)g * p.d3;
          const float* w4 = p.w4 + (size_t)g * p.d3;
          float e = 0.f;
          for (int cc = half; cc < p.d3 / 32; cc += 2) {
            float4 bb[8], ww[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              bb[k] = __ldg(reinterpret_cast<const float4*>(bias + cc * 32) + k);
              ww[k] = __ldg(reinterpret_cast<const float4*>(w4 + cc * 32) + k);
            }
            float v[32];
            tmem_ld32(tmem + b * 256 + lane_base + cc * 32, v);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
              const float zz[4] = {fmaf(v[4 * k], inv_s3, bb[k].x), fmaf(v[4 * k + 1], inv_s3, bb[k].y),
                                   fmaf(v[4 * k + 2], inv_s3, bb[k].z), fmaf(v[4 * k + 3], inv_s3, bb[k].w)};
              const float wv[4] = {ww[k].x, ww[k].y, ww[k].z, ww[k].w};
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                float h, dh;
                celu_pair(zz[u], p.alpha, celu_k2, h, dh);
                e = fmaf(h, wv[u], e);
                v[4 * k + u] = (s_g * wv[u]) * dh;
              }
            }
            act_store<F16>(act, r, cc * 32, v, grad_lo);
            publish_atom(cc >> 1);
          }
          release_acc(b);
          if (half == 1) {
            // the previous row energies must have been read before they are overwritten
            if (ex_phase > 0 && !(ok = wait_bar(&bars->ex_free, (ex_phase - 1) & 1, abort_flag, p.err, p.timeout_ns))) break;
            bars->ex[r] = e;
            mbar_arrive(&bars->ex_ready);
          } else {
            if (!(ok = wait_bar(&bars->ex_ready, ex_phase & 1, abort_flag, p.err, p.timeout_ns))) break;
            e += bars->ex[r] + __ldg(p.b4 + g);
            mbar_arrive(&bars->ex_free);
            e_row += e * p.inv_models;
            if (m == M - 1) p.e_rows[row] = e_row;
          }
          ++ex_phase;
        }
        // E4: G2 = D2 * celu'(z2) -> act
        {
          const uint32_t b = job & 1;
          if (!(ok = take_acc(b))) break;
          mask_layer(b, p.d2, p.d1);
          release_acc(b);
        }
        // E5: G1 = D1 * celu'(z1) -> act
        {
          const uint32_t b = job & 1;
          if (!(ok = take_acc(b))) break;
          mask_layer(b, p.d1, 0);
          release_acc(b);
        }
        // E6: dX chunks.  Each warp stages a 32 x 32 block (its 32 rows, 32
        // columns) in its own shared-memory tile, in the 128-byte-swizzled
        // layout of the dX tensor map, and the TMA engine writes it out: a bulk
        // store for the first model, a bulk FP32 add in the L2 for the others.
        // The lane that issues the copies first waits until its copies of the
        // previous model have completed, so every element sums the models in
        // model order.
        if (lane == 0) bulk_wait_all();
        __syncwarp();
        uint8_t* tile = reinterpret_cast<uint8_t*>(xpose + (warp - 2) * 32 * 32);
        uint8_t* trow = tile + lane * 128;
        const int dx_row = p.tile_row[w] + 32 * q;
        const float dx_scale = p.inv_models * (inv_s1 / s_g);
        for (int len = 0, c0 = run_at(p.kmask, 0, len); c0 >= 0 && ok; c0 = run_at(p.kmask, c0 + len, len)) {
          const uint32_t b = job & 1;
          if (!(ok = take_acc(b))) break;
          for (int cc = half; cc < 2 * len; cc += 2) {
            float v[32];
            tmem_ld32(tmem + b * 256 + lane_base + cc * 32, v);
            if (lane == 0) bulk_wait_read();  // the tile's previous copy has read it
            __syncwarp();
#pragma unroll
            for (int j = 0; j < 8; ++j)
              *reinterpret_cast<float4*>(trow + ((j ^ (lane & 7)) << 4)) =
                  make_float4(v[4 * j] * dx_scale, v[4 * j + 1] * dx_scale, v[4 * j + 2] * dx_scale,
                              v[4 * j + 3] * dx_scale);
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) {
              // the dE/dAEV block is added to once per model: kept in L2
              if (m == 0)
                tma_store_2d_hint(&maps.dx, tile, c0 * 64 + cc * 32, dx_row, l2_evict_last());
              else
                tma_add_2d_hint(&maps.dx, tile, c0 * 64 + cc * 32, dx_row, l2_evict_last());
              bulk_commit();
            }
          }
          release_acc(b);
        }
      }
    }
    // the dX copies have completed (and no longer read shared memory) before
    // the CTA exits
    if (lane == 0) bulk_wait_all();
    __syncwarp();
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    fence_after_sync();
    tmem_dealloc(tmem, 512);
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }
  return fn;
}

// 16-bit [rows][cols] operand (BF16, or FP16 when f16) in BK x box_rows boxes
bool map2d(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols, uint32_t box_rows, bool f16 = false) {
  auto fn = encode_fn();
  if (!fn || !base) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base),
            dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// dX as FP32 [rows][cols] in 32 x 32 boxes (128-byte rows, 128-byte swizzle)
bool map_dx(CUtensorMap* m, void* base, uint64_t rows, uint64_t cols) {
  auto fn = encode_fn();
  if (!fn || !base) return false;
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 4};
  cuuint32_t box[2] = {32, 32};
  cuuint32_t estr[2] = {1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
  }
  return n;
}

bool is_f16_form(int precision) {
  return precision == FENNOL_MLP_F16X3X1 || precision == FENNOL_MLP_F16X3X2;
}

}  // namespace

// Shape check: the fused kernel needs every hidden width <= 256 (activation
// buffer), the input width a multiple of 256 and a BF16, BF16x2 or FP16 form.
bool fnl_mlp_fused_supported(int precision, const fennol_mlp_weights* w) {
  const int* d = w->dims;
  if (precision != FENNOL_MLP_BF16 && precision != FENNOL_MLP_BF16X2 && !is_f16_form(precision)) return false;
  if (is_f16_form(precision) && !w->f16_scale) return false;
  if (d[0] % 256 != 0 || d[0] > 4096) return false;
  for (int l = 1; l < 4; ++l)
    if (d[l] > 256 || d[l] % 64 != 0) return false;
  return true;
}

size_t fnl_mlp_fused_workspace(const fennol_mlp_weights* w) {
  return 256 + 128 + (size_t)sm_count() * BM * (w->dims[1] + w->dims[2]) * sizeof(float);
}

int fnl_mlp_fused(int precision, int rows, int ntiles, const int* tile_species, const int* tile_row,
                  const fennol_mlp_weights* w, const void* x, const void* x_lo, unsigned long long kmask,
                  float* e_rows, float* dx, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (!encode_fn()) return FENNOL_ERR_UNSUPPORTED;
  if (ws_bytes < fnl_mlp_fused_workspace(w)) return FENNOL_ERR_WORKSPACE;
  const int* d = w->dims;
  const int G = w->n_models * w->n_species;
  const bool f16 = is_f16_form(precision);
  const bool alo = precision == FENNOL_MLP_BF16X2 || f16;
  const bool glo = precision == FENNOL_MLP_BF16X2;
  const bool wflo = f16;
  const bool wblo = precision == FENNOL_MLP_F16X3X2;
  if (f16 && (!w->wt_lo[0] || !w->wt_lo[1] || !w->wt_lo[2])) return FENNOL_ERR_INVALID;
  if (wblo && (!w->w_lo[0] || !w->w_lo[1] || !w->w_lo[2])) return FENNOL_ERR_INVALID;
  if (f16 && ((uintptr_t)w->f16_scale & 15) != 0) return FENNOL_ERR_INVALID;
  // maps of absent low parts alias the high parts (never loaded)
  const void* wtl[3] = {wflo ? w->wt_lo[0] : w->wt_hi[0], wflo ? w->wt_lo[1] : w->wt_hi[1],
                        wflo ? w->wt_lo[2] : w->wt_hi[2]};
  const void* wl[3] = {wblo ? w->w_lo[0] : w->w_hi[0], wblo ? w->w_lo[1] : w->w_hi[1],
                       wblo ? w->w_lo[2] : w->w_hi[2]};
  Maps maps;
  bool ok = map2d(&maps.x, x, rows, d[0], BM, f16) && map2d(&maps.xlo, alo ? x_lo : x, rows, d[0], BM, f16) &&
            map2d(&maps.w1t, w->wt_hi[0], (uint64_t)G * d[1], d[0], d[1], f16) &&
            map2d(&maps.w2t, w->wt_hi[1], (uint64_t)G * d[2], d[1], d[2], f16) &&
            map2d(&maps.w3t, w->wt_hi[2], (uint64_t)G * d[3], d[2], d[3], f16) &&
            map2d(&maps.w3, w->w_hi[2], (uint64_t)G * d[2], d[3], d[2], f16) &&
            map2d(&maps.w2, w->w_hi[1], (uint64_t)G * d[1], d[2], d[1], f16) &&
            map2d(&maps.w1, w->w_hi[0], (uint64_t)G * d[0], d[1], 64, f16) &&
            map2d(&maps.w1t_lo, wtl[0], (uint64_t)G * d[1], d[0], d[1], f16) &&
            map2d(&maps.w2t_lo, wtl[1], (uint64_t)G * d[2], d[1], d[2], f16) &&
            map2d(&maps.w3t_lo, wtl[2], (uint64_t)G * d[3], d[2], d[3], f16) &&
            map2d(&maps.w3_lo, wl[2], (uint64_t)G * d[2], d[3], d[2], f16) &&
            map2d(&maps.w2_lo, wl[1], (uint64_t)G * d[1], d[2], d[1], f16) &&
            map2d(&maps.w1_lo, wl[0], (uint64_t)G * d[0], d[1], 64, f16) && map_dx(&maps.dx, dx, rows, d[0]);
  if (!ok) return FENNOL_ERR_CUDA;
  FusedParams p{};
  p.ntiles = ntiles;
  p.n_models = w->n_models;
  p.n_species = w->n_species;
  p.tile_species = tile_species;
  p.tile_row = tile_row;
  p.d0 = d[0];
  p.d1 = d[1];
  p.d2 = d[2];
  p.d3 = d[3];
  p.a_lo = alo ? 1 : 0;
  p.g_lo = glo ? 1 : 0;
  p.wf_lo = wflo ? 1 : 0;
  p.wb_lo = wblo ? 1 : 0;
  p.xstages = wflo ? kXStagesWide : kXStages;
  p.xstage = wflo ? kXStageWide : kXStage;
  p.scales = reinterpret_cast<const float4*>(w->f16_scale);
  const int nck = d[0] / BK;
  p.kmask = kmask & (nck >= 64 ? ~0ull : ((1ull << nck) - 1));
  if (!p.kmask) return FENNOL_ERR_INVALID;
  p.alpha = w->celu_alpha;
  p.inv_models = 1.0f / (float)w->n_models;
  p.b1 = w->b32[0];
  p.b2 = w->b32[1];
  p.b3 = w->b32[2];
  p.w4 = w->w32[3];
  p.b4 = w->b32[3];
  p.e_rows = e_rows;
  p.dx = dx;
  p.err = (int*)ws;
  p.timeout_ns = g_wait_limit_ns;
  p.stall = 0;
  if (g_stall_launches > 0) {
    p.stall = 1;
    --g_stall_launches;
  }
  // CELU' scratch on a 128-byte boundary: its L2 lines are discarded whole
  p.dc = (float*)(((uintptr_t)ws + 256 + 127) & ~(uintptr_t)127);
  const size_t smem = kSmemMain + sizeof(Bars) + 1024;
  static bool attr[2] = {false, false};
  auto kern = f16 ? k_mlp_fused<true> : k_mlp_fused<false>;
  if (!attr[f16]) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
      return FENNOL_ERR_CUDA;
    attr[f16] = true;
  }
  if (ntiles <= 0) return FENNOL_OK;
  const int grid = ntiles < sm_count() ? ntiles : sm_count();
  FNL_LAUNCH_PDL(kern, dim3(grid), dim3(kThreads), smem, st, maps, p);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_mlp_wait_limit(double seconds) {
  if (!(seconds > 0.0) || seconds > 60.0) return FENNOL_ERR_INVALID;
  g_wait_limit_ns = (uint64_t)(seconds * 1e9);
  return FENNOL_OK;
}

extern "C" int fennol_mlp_inject_stall(int launches) {
  if (launches < 0) return FENNOL_ERR_INVALID;
  g_stall_launches = launches;
  return FENNOL_OK;
}
