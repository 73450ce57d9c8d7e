// Species-indexed MLP on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Replaces SpeciesIndexNet / FullyConnectedNet (src/fennol/models/misc/nets.py:
// 13-102, 301-426) and the transpose jax.grad builds for the input gradient.
// Six grouped GEMMs per model (3 forward, 3 input-gradient); each CTA computes
// one 128-row tile (one species) x up to 256 columns:
//   warp 0      TMA producer: A and B tiles (K-chunks of 64 bf16, 128-byte
//               swizzle) into a multi-stage shared-memory ring;
//   warp 1      allocates the TMEM accumulator, one thread issues
//               tcgen05.mma (M=128, N=bn, K=16) and tcgen05.commit;
//   warps 2-9   epilogue: tcgen05.ld of the FP32 accumulator (one row per
//               thread, two warps per TMEM lane quarter splitting the
//               columns), fused bias + CELU / CELU' / energy head, stores.
// Launches use programmatic dependent launch: a kernel's prologue (barrier
// init, TMEM allocation) and its first weight tiles overlap the tail of the
// previous kernel; inputs written by that kernel are read only after
// griddepcontrol.wait.
// Split-BF16 operands: activations are carried as hi + lo bfloat16 pairs
// (x = hi + lo to ~16 bits) and, in the 3-product form, weights too:
// acc += A_hi B_hi + A_lo B_hi (+ A_hi B_lo), all accumulated in FP32 TMEM.
// Every mbarrier wait is bounded by a 2 s deadline; on expiry the CTA sets the
// error word at the start of the workspace, finishes and frees its TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdlib>
#include <mutex>
#include <string>
#include <unordered_map>

#include "mlp_common.cuh"
#include "umma.cuh"

using namespace fnl;
using namespace fnl::umma;

namespace {

constexpr int kThreads = 320;
constexpr int kEpiThreads = 256;
constexpr int BM = 128, BK = 64;
constexpr uint64_t kTimeoutNs = 2000000000ull;
constexpr int kSmemBudget = 220 * 1024;

enum EpiKind { EPI_HIDDEN = 0, EPI_HEAD = 1, EPI_DACT = 2, EPI_OUT = 3 };

struct TcParams {
  int nk;                // K chunks of 64
  int bn;                // columns per work item (multiple of 32, <= 256)
  int n_chunks;          // work items per tile along N
  int b_group_rows;      // rows of the B matrix per group
  int n_full;            // full output width (bias/w4 stride)
  int group0;            // model * n_species
  const int* tile_species;
  const int* tile_row;
  int a_lo, b_lo;        // split operands present
  int stages;
  uint32_t tmem_cols;
  const float* bias;     // [G][n_full]
  const float* w4;       // [G][n_full] (EPI_HEAD)
  const float* b4;       // [G]
  float alpha;
  float inv_models;
  int first_model;
  __nv_bfloat16* out_hi;
  __nv_bfloat16* out_lo;
  int ld_out;
  const __nv_bfloat16* act_hi;  // EPI_DACT: forward activation of this layer
  const __nv_bfloat16* act_lo;
  float* e_part;        // EPI_HEAD: [slot][rows] partial energies (slot = model*n_chunks + chunk)
  int slot_base;
  int rows;
  float* out_f32;
  int ld_f32;
  int* err;
};

__device__ __forceinline__ float dcelu_from_z(float z, float alpha) { return z > 0.f ? 1.f : __expf(z / alpha); }
__device__ __forceinline__ float celu_fast(float x, float alpha) {
  return x > 0.f ? x : alpha * (__expf(x / alpha) - 1.f);
}
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void epi_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kEpiThreads) : "memory"); }

__device__ __forceinline__ void split_store(__nv_bfloat16* hi, __nv_bfloat16* lo, const float* v) {
  // 32 values -> 64 bytes of hi (and lo) as four 16-byte stores each
  uint32_t h[16], l[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    __nv_bfloat16 a = __float2bfloat16_rn(v[2 * k]), b = __float2bfloat16_rn(v[2 * k + 1]);
    h[k] = (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
    if (lo) {
      __nv_bfloat16 c = __float2bfloat16_rn(v[2 * k] - __bfloat162float(a));
      __nv_bfloat16 d = __float2bfloat16_rn(v[2 * k + 1] - __bfloat162float(b));
      l[k] = (uint32_t)__bfloat16_as_ushort(c) | ((uint32_t)__bfloat16_as_ushort(d) << 16);
    }
  }
  uint4* ph = reinterpret_cast<uint4*>(hi);
#pragma unroll
  for (int q = 0; q < 4; ++q) ph[q] = make_uint4(h[4 * q], h[4 * q + 1], h[4 * q + 2], h[4 * q + 3]);
  if (lo) {
    uint4* pl = reinterpret_cast<uint4*>(lo);
#pragma unroll
    for (int q = 0; q < 4; ++q) pl[q] = make_uint4(l[4 * q], l[4 * q + 1], l[4 * q + 2], l[4 * q + 3]);
  }
}

__device__ __forceinline__ void load_bf16x32(const __nv_bfloat16* p, float* v) {
  const uint4* q = reinterpret_cast<const uint4*>(p);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    uint4 u = q[k];
    uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[8 * k + 2 * j] = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w[j] & 0xFFFF)));
      v[8 * k + 2 * j + 1] = __bfloat162float(__ushort_as_bfloat16((unsigned short)(w[j] >> 16)));
    }
  }
}

template <int EPI>
__global__ void __launch_bounds__(kThreads, 1)
k_umma_gemm(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapAlo,
            const __grid_constant__ CUtensorMap mapB, const __grid_constant__ CUtensorMap mapBlo,
            const TcParams p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t a_bytes = BM * BK * 2;
  const uint32_t b_bytes = (uint32_t)p.bn * BK * 2;
  const uint32_t stage_bytes = a_bytes * (1 + p.a_lo) + b_bytes * (1 + p.b_lo);
  uint64_t* full = (uint64_t*)(smem + (size_t)p.stages * stage_bytes);
  uint64_t* empty = full + p.stages;
  uint64_t* accum = empty + p.stages;
  uint32_t* tmem_slot = (uint32_t*)(accum + 1);

  const int tile = blockIdx.x / p.n_chunks;
  const int chunk = blockIdx.x % p.n_chunks;
  const int a_row = p.tile_row[tile];
  const int grp = p.group0 + p.tile_species[tile];
  const int b_row = grp * p.b_group_rows + chunk * p.bn;
  const int n0 = chunk * p.bn;
  const uint64_t deadline = globaltimer() + kTimeoutNs;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.stages; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, 1);
    }
    mbar_init(accum, 1);
    fence_barrier_init();
    prefetch_tensormap(&mapA);
    prefetch_tensormap(&mapB);
  }
  if (warp == 1) tmem_alloc(tmem_slot, p.tmem_cols);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  bool failed = false;
  griddep_launch();

  auto stage_a = [&](int s) { return smem + (size_t)s * stage_bytes; };
  auto stage_alo = [&](int s) { return smem + (size_t)s * stage_bytes + a_bytes; };
  auto stage_b = [&](int s) { return smem + (size_t)s * stage_bytes + a_bytes * (1 + p.a_lo); };
  auto stage_blo = [&](int s) { return stage_b(s) + b_bytes; };

  if (warp == 0) {
    if (lane == 0) {
      // weights do not depend on the previous kernel: fetch the first stages now
      const int pre = p.nk < p.stages ? p.nk : p.stages;
      for (int kc = 0; kc < pre; ++kc) {
        mbar_expect_tx(full + kc, stage_bytes);
        tma_load_2d(&mapB, full + kc, stage_b(kc), kc * BK, b_row);
        if (p.b_lo) tma_load_2d(&mapBlo, full + kc, stage_blo(kc), kc * BK, b_row);
      }
      griddep_wait();
      for (int kc = 0; kc < pre; ++kc) {
        tma_load_2d(&mapA, full + kc, stage_a(kc), kc * BK, a_row);
        if (p.a_lo) tma_load_2d(&mapAlo, full + kc, stage_alo(kc), kc * BK, a_row);
      }
      for (int kc = pre; kc < p.nk; ++kc) {
        int s = kc % p.stages, u = kc / p.stages;
        if (!mbar_wait(empty + s, (u - 1) & 1, deadline)) {
          failed = true;
          break;
        }
        mbar_expect_tx(full + s, stage_bytes);
        tma_load_2d(&mapA, full + s, stage_a(s), kc * BK, a_row);
        if (p.a_lo) tma_load_2d(&mapAlo, full + s, stage_alo(s), kc * BK, a_row);
        tma_load_2d(&mapB, full + s, stage_b(s), kc * BK, b_row);
        if (p.b_lo) tma_load_2d(&mapBlo, full + s, stage_blo(s), kc * BK, b_row);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16_f32(p.bn);
      for (int kc = 0; kc < p.nk; ++kc) {
        int s = kc % p.stages, u = kc / p.stages;
        if (!mbar_wait(full + s, u & 1, deadline)) {
          failed = true;
          break;
        }
        fence_after_sync();
        const uint32_t sa = smem_u32(stage_a(s)), sal = smem_u32(stage_alo(s));
        const uint32_t sb = smem_u32(stage_b(s)), sbl = smem_u32(stage_blo(s));
#pragma unroll
        for (int kk = 0; kk < BK / 16; ++kk) {
          uint64_t ad = sdesc_sw128(sa + kk * 32), bd = sdesc_sw128(sb + kk * 32);
          mma_bf16(tmem, ad, bd, idesc, (kc | kk) != 0);
          if (p.a_lo) mma_bf16(tmem, sdesc_sw128(sal + kk * 32), bd, idesc, 1u);
          if (p.b_lo) mma_bf16(tmem, ad, sdesc_sw128(sbl + kk * 32), idesc, 1u);
        }
        mma_commit(empty + s);
      }
      mma_commit(accum);
    }
  } else {
    // epilogue: 8 warps; TMEM lane quarter = warp % 4, column half = (warp - 2) / 4
    const int q = warp & 3;
    const int half = (warp - 2) >> 2;
    const int r = 32 * q + lane;
    const int row = a_row + r;
    griddep_wait();
    // warp-uniform decision: tcgen05.ld below is a warp-collective instruction
    const bool ready = __all_sync(0xffffffffu, mbar_wait(accum, 0, deadline));
    float e = 0.f;
    if (!ready) {
      failed = true;
    } else {
      fence_after_sync();
      const float* bias = p.bias ? p.bias + (size_t)grp * p.n_full : nullptr;
      const float* w4 = p.w4 ? p.w4 + (size_t)grp * p.n_full : nullptr;
      for (int cc = half; cc < p.bn / 32; cc += 2) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(cc * 32), v);
        const int n = n0 + cc * 32;
        if (EPI == EPI_HIDDEN) {
#pragma unroll
          for (int k = 0; k < 32; ++k) v[k] = celu_fast(v[k] + __ldg(bias + n + k), p.alpha);
          split_store(p.out_hi + (size_t)row * p.ld_out + n,
                      p.out_lo ? p.out_lo + (size_t)row * p.ld_out + n : nullptr, v);
        } else if (EPI == EPI_HEAD) {
#pragma unroll
          for (int k = 0; k < 32; ++k) {
            float z = v[k] + __ldg(bias + n + k);
            float wv = __ldg(w4 + n + k);
            e = fmaf(celu_fast(z, p.alpha), wv, e);
            v[k] = wv * dcelu_from_z(z, p.alpha);
          }
          split_store(p.out_hi + (size_t)row * p.ld_out + n,
                      p.out_lo ? p.out_lo + (size_t)row * p.ld_out + n : nullptr, v);
        } else if (EPI == EPI_DACT) {
          float h[32], hl[32];
          load_bf16x32(p.act_hi + (size_t)row * p.ld_out + n, h);
          if (p.act_lo) {
            load_bf16x32(p.act_lo + (size_t)row * p.ld_out + n, hl);
#pragma unroll
            for (int k = 0; k < 32; ++k) h[k] += hl[k];
          }
#pragma unroll
          for (int k = 0; k < 32; ++k) v[k] *= dcelu_from_h(h[k], p.alpha);
          split_store(p.out_hi + (size_t)row * p.ld_out + n,
                      p.out_lo ? p.out_lo + (size_t)row * p.ld_out + n : nullptr, v);
        } else {  // EPI_OUT
          float4* o = reinterpret_cast<float4*>(p.out_f32 + (size_t)row * p.ld_f32 + n);
#pragma unroll
          for (int k = 0; k < 8; ++k) {
            float4 a = make_float4(v[4 * k] * p.inv_models, v[4 * k + 1] * p.inv_models,
                                   v[4 * k + 2] * p.inv_models, v[4 * k + 3] * p.inv_models);
            if (!p.first_model) {
              float4 b = o[k];
              a.x += b.x;
              a.y += b.y;
              a.z += b.z;
              a.w += b.w;
            }
            o[k] = a;
          }
        }
      }
    }
    if (EPI == EPI_HEAD) {
      // combine the two column halves of this row, then one partial per (model, chunk)
      float* ex = reinterpret_cast<float*>(tmem_slot + 4);
      if (half == 1) ex[r] = e;
      epi_bar();
      if (half == 0 && ready) {
        e += ex[r];
        if (chunk == 0) e += __ldg(p.b4 + grp);
        p.e_part[(size_t)(p.slot_base + chunk) * p.rows + row] = e;
      }
    }
  }
  if (failed) atomicExch(p.err, 1);
  fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    fence_after_sync();
    tmem_dealloc(tmem, p.tmem_cols);
  }
}

// ------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  });
  return fn;
}

// 2-D bf16 K-major map [rows][cols] with a (64 x box_rows) box, 128-byte swizzle.
bool make_map(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols, uint32_t box_rows) {
  auto fn = encode_fn();
  if (!fn || !base) return false;
  static std::mutex mu;
  static std::unordered_map<std::string, CUtensorMap> cache;
  std::string key((const char*)&base, sizeof(base));
  key.append((const char*)&rows, sizeof(rows));
  key.append((const char*)&cols, sizeof(cols));
  key.append((const char*)&box_rows, sizeof(box_rows));
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(key);
    if (it != cache.end()) {
      *m = it->second;
      return true;
    }
  }
  cuuint64_t dims[2] = {cols, rows};
  cuuint64_t strides[1] = {cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)BK, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return false;
  std::lock_guard<std::mutex> g(mu);
  if (cache.size() > 4096) cache.clear();
  cache[key] = *m;
  return true;
}

struct Gemm {
  const void* a;
  const void* a_lo;
  int lda;  // columns of A (= K)
  const void* b;
  const void* b_lo;
  int b_total_rows;
  int K, N, bn;
  int epi;
  TcParams p;
};

template <int EPI>
int launch_epi(const Gemm& g, int rows, int ntiles, cudaStream_t st) {
  CUtensorMap ma, mal, mb, mbl;
  if (!make_map(&ma, g.a, rows, g.K, BM)) return FENNOL_ERR_CUDA;
  if (!make_map(&mal, g.a_lo ? g.a_lo : g.a, rows, g.K, BM)) return FENNOL_ERR_CUDA;
  if (!make_map(&mb, g.b, g.b_total_rows, g.K, g.bn)) return FENNOL_ERR_CUDA;
  if (!make_map(&mbl, g.b_lo ? g.b_lo : g.b, g.b_total_rows, g.K, g.bn)) return FENNOL_ERR_CUDA;
  TcParams p = g.p;
  uint32_t stage = (uint32_t)BM * BK * 2 * (1 + p.a_lo) + (uint32_t)g.bn * BK * 2 * (1 + p.b_lo);
  int stages = (int)((kSmemBudget - 2048) / stage);
  if (stages > 4) stages = 4;
  if (stages < 2) return FENNOL_ERR_UNSUPPORTED;
  p.stages = stages;
  uint32_t cols = 32;
  while (cols < (uint32_t)g.bn) cols <<= 1;
  p.tmem_cols = cols;
  size_t smem = (size_t)stages * stage + 1024 + 1024;
  static bool attr_set = false;
  if (!attr_set) {
    if (cudaFuncSetAttribute(k_umma_gemm<EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBudget + 2048) !=
        cudaSuccess)
      return FENNOL_ERR_CUDA;
    attr_set = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ntiles * p.n_chunks);
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, k_umma_gemm<EPI>, ma, mal, mb, mbl, p) != cudaSuccess) return FENNOL_ERR_CUDA;
  return FENNOL_OK;
}

int launch(const Gemm& g, int rows, int ntiles, cudaStream_t st) {
  switch (g.epi) {
    case EPI_HIDDEN: return launch_epi<EPI_HIDDEN>(g, rows, ntiles, st);
    case EPI_HEAD: return launch_epi<EPI_HEAD>(g, rows, ntiles, st);
    case EPI_DACT: return launch_epi<EPI_DACT>(g, rows, ntiles, st);
    default: return launch_epi<EPI_OUT>(g, rows, ntiles, st);
  }
}

struct TcWs {
  int* err;
  __nv_bfloat16 *h1, *h1l, *h2, *h2l, *g3, *g3l;
  float* e_part;  // [n_models * kHeadChunks][rows]
};

constexpr int kHeadChunks = 2;

// e_rows[r] = sum over (model, chunk) partials / n_models, fixed order.
__global__ void k_e_rows(const float* __restrict__ e_part, int slots, int rows, float inv_models,
                         float* __restrict__ e_rows) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  float e = 0.f;
  for (int k = 0; k < slots; ++k) e += e_part[(size_t)k * rows + r];
  e_rows[r] = e * inv_models;
}

size_t tc_layout(int rows, const fennol_mlp_weights* w, char* base, TcWs* out) {
  const size_t ep = (size_t)w->n_models * kHeadChunks * rows * sizeof(float);
  size_t off = 256;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = (off + bytes + 1023) / 1024 * 1024;
    return o;
  };
  size_t d1 = (size_t)rows * w->dims[1] * 2, d2 = (size_t)rows * w->dims[2] * 2,
         d3 = (size_t)rows * w->dims[3] * 2;
  size_t o1 = take(d1), o1l = take(d1), o2 = take(d2), o2l = take(d2), o3 = take(d3), o3l = take(d3);
  size_t oe = take(ep);
  if (base && out) {
    out->err = (int*)base;
    out->h1 = (__nv_bfloat16*)(base + o1);
    out->h1l = (__nv_bfloat16*)(base + o1l);
    out->h2 = (__nv_bfloat16*)(base + o2);
    out->h2l = (__nv_bfloat16*)(base + o2l);
    out->g3 = (__nv_bfloat16*)(base + o3);
    out->g3l = (__nv_bfloat16*)(base + o3l);
    out->e_part = (float*)(base + oe);
  }
  return off;
}

}  // namespace

size_t fnl_mlp_tc_workspace(int precision, int rows, int n_models, const fennol_mlp_weights* w) {
  (void)n_models;
  size_t a = tc_layout(rows, w, nullptr, nullptr);
  if (fnl_mlp_fused_supported(precision, w)) {
    size_t b = fnl_mlp_fused_workspace(w);
    if (b > a) a = b;
  }
  return a;
}

int fnl_mlp_tc(int precision, int rows, int ntiles, const int* tile_species, const int* tile_row,
               const fennol_mlp_weights* w, const void* x, const void* x_lo, unsigned long long kmask,
               float* e_rows, float* dx, void* ws, size_t ws_bytes, cudaStream_t st) {
  if (!encode_fn()) return FENNOL_ERR_UNSUPPORTED;
  const bool f16 = precision == FENNOL_MLP_F16X3X1 || precision == FENNOL_MLP_F16X3X2;
  if (fnl_mlp_fused_supported(precision, w) && (f16 || !getenv("FENNOL_MLP_UNFUSED")))
    return fnl_mlp_fused(precision, rows, ntiles, tile_species, tile_row, w, x, x_lo, kmask, e_rows, dx, ws,
                         ws_bytes, st);
  if (f16) return FENNOL_ERR_UNSUPPORTED;  // the FP16 forms exist only as the fused kernel
  const int* d = w->dims;
  for (int l = 0; l < 4; ++l)
    if (d[l] > 1024 || (l > 0 && d[l] > 256)) return FENNOL_ERR_UNSUPPORTED;
  if (ws_bytes < tc_layout(rows, w, nullptr, nullptr)) return FENNOL_ERR_WORKSPACE;
  TcWs t;
  tc_layout(rows, w, (char*)ws, &t);
  const bool alo = precision != FENNOL_MLP_BF16;
  const bool blo = precision == FENNOL_MLP_BF16X3;
  if (!alo) {
    t.h1l = t.h2l = t.g3l = nullptr;
  }
  const int G = w->n_models * w->n_species;
  const float inv_m = 1.0f / (float)w->n_models;
  auto base = [&](int epi, const void* a, const void* al, int K, const void* b, const void* bl, int b_group_rows,
                  int N, int bn, int g0) {
    Gemm g{};
    g.a = a;
    g.a_lo = alo ? al : nullptr;
    g.lda = K;
    g.b = b;
    g.b_lo = blo ? bl : nullptr;
    g.b_total_rows = G * b_group_rows;
    g.K = K;
    g.N = N;
    g.bn = bn;
    g.epi = epi;
    TcParams& p = g.p;
    p.nk = K / BK;
    p.bn = bn;
    p.n_chunks = N / bn;
    p.b_group_rows = b_group_rows;
    p.n_full = N;
    p.group0 = g0;
    p.tile_species = tile_species;
    p.tile_row = tile_row;
    p.a_lo = alo ? 1 : 0;
    p.b_lo = blo ? 1 : 0;
    p.alpha = w->celu_alpha;
    p.inv_models = inv_m;
    p.err = t.err;
    return g;
  };
  for (int m = 0; m < w->n_models; ++m) {
    const int g0 = m * w->n_species;
    int rc;
    // L1: H1 = celu(X W1 + b1)
    Gemm g = base(EPI_HIDDEN, x, x_lo, d[0], w->wt_hi[0], w->wt_lo[0], d[1], d[1], d[1] / 2, g0);
    g.p.bias = w->b32[0];
    g.p.out_hi = t.h1;
    g.p.out_lo = t.h1l;
    g.p.ld_out = d[1];
    if ((rc = launch(g, rows, ntiles, st))) return rc;
    // L2: H2 = celu(H1 W2 + b2)
    g = base(EPI_HIDDEN, t.h1, t.h1l, d[1], w->wt_hi[1], w->wt_lo[1], d[2], d[2], d[2] / 2, g0);
    g.p.bias = w->b32[1];
    g.p.out_hi = t.h2;
    g.p.out_lo = t.h2l;
    g.p.ld_out = d[2];
    if ((rc = launch(g, rows, ntiles, st))) return rc;
    // L3 + head: e = celu(H2 W3 + b3) . w4 + b4 ; G3 = w4 * celu'(z3)
    g = base(EPI_HEAD, t.h2, t.h2l, d[2], w->wt_hi[2], w->wt_lo[2], d[3], d[3], d[3] / kHeadChunks, g0);
    g.p.bias = w->b32[2];
    g.p.w4 = w->w32[3];
    g.p.b4 = w->b32[3];
    g.p.out_hi = t.g3;
    g.p.out_lo = t.g3l;
    g.p.ld_out = d[3];
    g.p.e_part = t.e_part;
    g.p.slot_base = m * kHeadChunks;
    g.p.rows = rows;
    g.p.first_model = m == 0;
    if ((rc = launch(g, rows, ntiles, st))) return rc;
    // B3: G2 = (G3 W3^T) * celu'(H2), in place of H2
    g = base(EPI_DACT, t.g3, t.g3l, d[3], w->w_hi[2], w->w_lo[2], d[2], d[2], d[2] / 2, g0);
    g.p.act_hi = t.h2;
    g.p.act_lo = t.h2l;
    g.p.out_hi = t.h2;
    g.p.out_lo = t.h2l;
    g.p.ld_out = d[2];
    if ((rc = launch(g, rows, ntiles, st))) return rc;
    // B2: G1 = (G2 W2^T) * celu'(H1), in place of H1
    g = base(EPI_DACT, t.h2, t.h2l, d[2], w->w_hi[1], w->w_lo[1], d[1], d[1], d[1] / 2, g0);
    g.p.act_hi = t.h1;
    g.p.act_lo = t.h1l;
    g.p.out_hi = t.h1;
    g.p.out_lo = t.h1l;
    g.p.ld_out = d[1];
    if ((rc = launch(g, rows, ntiles, st))) return rc;
    // B1: dX (+)= (G1 W1^T) / n_models
    g = base(EPI_OUT, t.h1, t.h1l, d[1], w->w_hi[0], w->w_lo[0], d[0], d[0], 128, g0);
    g.p.out_f32 = dx;
    g.p.ld_f32 = d[0];
    g.p.first_model = m == 0;
    if ((rc = launch(g, rows, ntiles, st))) return rc;
  }
  k_e_rows<<<(rows + 255) / 256, 256, 0, st>>>(t.e_part, w->n_models * kHeadChunks, rows, inv_m, e_rows);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}
