// Energy reduction, force output and the float64 MD integrator step.
//
// fennol_energy_reduce replaces the per-system segment_sum of
// FENNIX.total_energy (src/fennol/models/fennix.py:218-258) with a float64,
// fixed-order reduction.  fennol_md_step is the integrate() step of
// src/fennol/md/integrate.py:286-294 with the Langevin O step of
// src/fennol/md/thermostats.py:56-120 (NVE, :172-190, when a2 is NULL),
// carried in float64 and kept on the device.
#include <cmath>

#include "common.cuh"

using namespace fnl;

namespace {

// Fixed-order reduction in one launch.  System b (atoms sys_start[b] ..
// sys_start[b+1]) is cut into C_b = max(1, ceil(n_b / 1024)) chunks that start
// at its first atom; chunk c of system b owns the slot
//     base(b) + c,   base(b) = b + floor(sys_start[b] / 1024).
// base() is strictly increasing and base(b) + C_b <= base(b + 1), so slots
// are distinct without a prefix sum; a block finds the system of a slot by
// binary search on sys_start alone (slots past C_b are gaps).  Blocks write
// one float64 partial per chunk; the last block to finish (ticket counter)
// adds each system's partials in chunk order.  The result depends only on a
// system's own atoms, not on the rest of the batch.
constexpr int kRedChunk = 1024;

__device__ __forceinline__ int red_base(const int* sys_start, int b) { return b + sys_start[b] / kRedChunk; }
__device__ __forceinline__ int red_chunks(const int* sys_start, int b) {
  return max(1, (sys_start[b + 1] - sys_start[b] + kRedChunk - 1) / kRedChunk);
}

__global__ void __launch_bounds__(256) k_energy_sum(const float* __restrict__ e_rows, const int* __restrict__ atom_row,
                                                   const int* __restrict__ sys_start, int nsys, int nslots, double scale,
                                                   double* __restrict__ partial, double* __restrict__ e_atom,
                                                   double* __restrict__ energy, unsigned* __restrict__ ticket) {
  pdl_wait();
  __shared__ double part[256];
  __shared__ bool last;
  for (int w = blockIdx.x; w < nslots; w += gridDim.x) {
    // the system b with base(b) <= w < base(b + 1)
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (red_base(sys_start, mid) <= w) lo = mid; else hi = mid - 1;
    }
    const int b = lo, c = w - red_base(sys_start, b);
    if (c < 0 || c >= red_chunks(sys_start, b)) continue;  // a gap slot (uniform per block)
    const int i0 = sys_start[b] + c * kRedChunk;
    const int i1 = min(i0 + kRedChunk, sys_start[b + 1]);
    double s = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
      double e = scale * (double)e_rows[atom_row[i]];
      if (e_atom) e_atom[i] = e;
      s += e;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) partial[w] = part[0];
    __syncthreads();
  }
  // the last block to arrive sums the partials (all written before its ticket)
  __threadfence();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int b = threadIdx.x; b < nsys; b += blockDim.x) {
    const int base = red_base(sys_start, b), nc = red_chunks(sys_start, b);
    double s = 0.0;
    for (int k = 0; k < nc; ++k) s += __ldcg(partial + base + k);
    energy[b] = s;
  }
  if (threadIdx.x == 0) *ticket = 0u;  // ready for the next call
}

__global__ void k_forces_finalize(const float4* __restrict__ f4, int n, float scale, float* __restrict__ f) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = f4[i];
  f[3 * i] = scale * v.x;
  f[3 * i + 1] = scale * v.y;
  f[3 * i + 2] = scale * v.z;
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11).
struct U4 {
  unsigned x, y, z, w;
};
__device__ __forceinline__ U4 philox4x32_10(U4 c, unsigned k0, unsigned k1) {
  const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const unsigned W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    unsigned hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    unsigned hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// Box-Muller on two 32-bit uniforms -> two standard normals (float64).
__device__ __forceinline__ void box_muller(unsigned a, unsigned b, double& z0, double& z1) {
  double u1 = ((double)a + 1.0) * (1.0 / 4294967296.0);  // (0, 1]
  double u2 = (double)b * (1.0 / 4294967296.0);          // [0, 1)
  double r = sqrt(-2.0 * log(u1));
  double s, c;
  sincospi(2.0 * u2, &s, &c);
  z0 = r * c;
  z1 = r * s;
}

// One BAOAB update of atom i; `key`/`ctr` select its Philox noise block.
__device__ __forceinline__ void md_update(int i, double dt, double* __restrict__ x, double* __restrict__ v,
                                          const double* __restrict__ inv_mass, const float4* __restrict__ f4,
                                          double fscale, double a1, const double* __restrict__ a2,
                                          unsigned long long key, U4 ctr, float* __restrict__ coords,
                                          const int* __restrict__ sp, float4* __restrict__ xyzs,
                                          const double* __restrict__ x_ref, double half_skin2,
                                          int* rebuild_flag) {
  float4 f = f4[i];
  double im = inv_mass[i];
  double vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
  double px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
  // B: v += dt/m F
  vx += dt * im * (fscale * (double)f.x);
  vy += dt * im * (fscale * (double)f.y);
  vz += dt * im * (fscale * (double)f.z);
  // A: x += dt/2 v
  double h = 0.5 * dt;
  px += h * vx;
  py += h * vy;
  pz += h * vz;
  // O: Langevin
  if (a2) {
    U4 r = philox4x32_10(ctr, (unsigned)(key & 0xffffffffull), (unsigned)(key >> 32));
    double z0, z1, z2, z3;
    box_muller(r.x, r.y, z0, z1);
    box_muller(r.z, r.w, z2, z3);
    double s = a2[i];
    vx = a1 * vx + s * z0;
    vy = a1 * vy + s * z1;
    vz = a1 * vz + s * z2;
  }
  // A: x += dt/2 v
  px += h * vx;
  py += h * vy;
  pz += h * vz;
  v[3 * i] = vx;
  v[3 * i + 1] = vy;
  v[3 * i + 2] = vz;
  x[3 * i] = px;
  x[3 * i + 1] = py;
  x[3 * i + 2] = pz;
  float fx = (float)px, fy = (float)py, fz = (float)pz;
  if (coords) {
    coords[3 * i] = fx;
    coords[3 * i + 1] = fy;
    coords[3 * i + 2] = fz;
  }
  if (xyzs) xyzs[i] = make_float4(fx, fy, fz, __int_as_float(sp[i]));
  if (rebuild_flag && x_ref) {
    double dx = px - x_ref[3 * i], dy = py - x_ref[3 * i + 1], dz = pz - x_ref[3 * i + 2];
    if (dx * dx + dy * dy + dz * dz > half_skin2) *rebuild_flag = 1;
  }
}

__global__ void k_md_step(int n, double dt, double* __restrict__ x, double* __restrict__ v,
                          const double* __restrict__ inv_mass, const float4* __restrict__ f4,
                          double fscale, double a1, const double* __restrict__ a2,
                          unsigned long long seed, const unsigned long long* __restrict__ step_counter,
                          float* __restrict__ coords,
                          const int* __restrict__ sp, float4* __restrict__ xyzs,
                          const double* __restrict__ x_ref, double half_skin2, int* rebuild_flag) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long step = a2 ? *step_counter : 0ull;
  U4 ctr{(unsigned)i, (unsigned)(step & 0xffffffffull), (unsigned)(step >> 32), 0x4C47u};
  md_update(i, dt, x, v, inv_mass, f4, fscale, a1, a2, seed, ctr, coords, sp, xyzs, x_ref, half_skin2,
            rebuild_flag);
}

// Per-system noise streams: atom i of system b draws from the block keyed by
// sys_seed[b] at counter (i - sys_start[b], sys_step[b]), so a system's
// trajectory does not depend on which other systems share the batch.
__global__ void k_md_step_systems(int n, double dt, double* __restrict__ x, double* __restrict__ v,
                                  const double* __restrict__ inv_mass, const float4* __restrict__ f4,
                                  double fscale, double a1, const double* __restrict__ a2,
                                  const int* __restrict__ atom_sys, const int* __restrict__ sys_start,
                                  const unsigned long long* __restrict__ sys_seed,
                                  const unsigned long long* __restrict__ sys_step, float* __restrict__ coords,
                                  const int* __restrict__ sp, float4* __restrict__ xyzs,
                                  const double* __restrict__ x_ref, double half_skin2, int* rebuild_flag) {
  pdl_wait();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = atom_sys[i];
  const unsigned long long step = sys_step[b];
  U4 ctr{(unsigned)(i - sys_start[b]), (unsigned)(step & 0xffffffffull), (unsigned)(step >> 32), 0x4C47u};
  md_update(i, dt, x, v, inv_mass, f4, fscale, a1, a2, sys_seed[b], ctr, coords, sp, xyzs, x_ref,
            half_skin2, rebuild_flag);
}

__global__ void k_inc_steps(int nsys, unsigned long long* __restrict__ sys_step) {
  pdl_wait();
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nsys) sys_step[b] += 1ull;
}

__global__ void k_inc_counter(unsigned long long* c) {
  pdl_wait(); *c += 1ull; }

__global__ void k_mark_rebuilt(int n, const double* __restrict__ x, double* __restrict__ x_ref, int* flag) {
  pdl_wait();
  if (*flag == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 3 * n) x_ref[i] = x[i];
}
__global__ void k_clear_flag(int* flag) {
  pdl_wait(); *flag = 0; }

__global__ void k_kinetic(int n, const double* __restrict__ v, const double* __restrict__ inv_mass,
                          double* out) {
  pdl_wait();
  __shared__ double part[1024];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double vx = v[3 * i], vy = v[3 * i + 1], vz = v[3 * i + 2];
    s += (vx * vx + vy * vy + vz * vz) / inv_mass[i];
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = 0.5 * part[0];
}

}  // namespace

extern "C" size_t fennol_energy_workspace_bytes(int natoms, int nsys) {
  if (natoms < 0 || nsys < 0) return 0;
  size_t slots = (size_t)natoms / kRedChunk + (size_t)nsys + 1;
  return 256 + slots * sizeof(double);
}

// Per-system sum of per-centre virials, fixed order (one block per system).
__global__ void __launch_bounds__(256) k_virial_reduce(const float* __restrict__ av,
                                                       const int* __restrict__ sys_start, double scale,
                                                       double* __restrict__ vir) {
  pdl_wait();
  __shared__ double red[9][256];
  const int b = blockIdx.x, tid = threadIdx.x;
  double acc[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) acc[q] = 0.0;
  for (int i = sys_start[b] + tid; i < sys_start[b + 1]; i += 256)
#pragma unroll
    for (int q = 0; q < 9; ++q) acc[q] += (double)av[(size_t)i * 9 + q];
#pragma unroll
  for (int q = 0; q < 9; ++q) red[q][tid] = acc[q];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (tid < w)
#pragma unroll
      for (int q = 0; q < 9; ++q) red[q][tid] += red[q][tid + w];
    __syncthreads();
  }
  if (tid < 9) vir[(size_t)b * 9 + tid] = scale * red[tid][0];
}

extern "C" int fennol_virial_reduce(const float* atom_virial, int natoms, const int* sys_start, int nsys,
                                    double scale, double* virial, void* stream) {
  if (natoms < 0 || nsys < 0) return FENNOL_ERR_INVALID;
  if (nsys == 0) return FENNOL_OK;
  if (!sys_start || !virial || (natoms > 0 && !atom_virial)) return FENNOL_ERR_INVALID;
  FNL_LAUNCH_PDL(k_virial_reduce, nsys, 256, 0, (cudaStream_t)stream, atom_virial, sys_start, scale, virial);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_energy_reduce(const float* e_rows, const int* atom_row, int natoms,
                                    const int* sys_start, int nsys, double scale, double* energy,
                                    double* e_atom, void* workspace, size_t workspace_bytes,
                                    void* stream) {
  if (natoms < 0 || nsys < 0) return FENNOL_ERR_INVALID;
  if (nsys == 0) return FENNOL_OK;
  if (!sys_start || !energy || !workspace || (natoms > 0 && (!e_rows || !atom_row))) return FENNOL_ERR_INVALID;
  if (workspace_bytes < fennol_energy_workspace_bytes(natoms, nsys)) return FENNOL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned* ticket = (unsigned*)workspace;
  double* partial = (double*)((char*)workspace + 256);
  // slots: base(nsys - 1) + C_{nsys-1} <= nsys + natoms / 1024 + 1
  const int nslots = natoms / kRedChunk + nsys + 1;
  const int blocks = nslots < 4 * 148 ? nslots : 4 * 148;
  FNL_LAUNCH_PDL(k_energy_sum, blocks, 256, 0, st, e_rows, atom_row, sys_start, nsys, nslots, scale, partial, e_atom,
                 energy, ticket);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_forces_finalize(const float* forces4, int natoms, float scale, float* forces,
                                      void* stream) {
  if (natoms < 0) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!forces4 || !forces) return FENNOL_ERR_INVALID;
  FNL_LAUNCH_PDL(k_forces_finalize, (natoms + 255) / 256, 256, 0, (cudaStream_t)stream, (const float4*)forces4, natoms,
                                                                             scale, forces);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_md_step(int natoms, double dt, double* x, double* v, const double* inv_mass,
                              const float* forces4, double force_scale, double a1, const double* a2,
                              unsigned long long seed, unsigned long long* step_counter,
                              float* coords, const int* species_idx, float* xyzs,
                              const double* x_ref, double half_skin, int* rebuild_flag,
                              void* stream) {
  if (natoms < 0 || !(dt > 0)) return FENNOL_ERR_INVALID;
  if (a2 && !step_counter) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!x || !v || !inv_mass || !forces4) return FENNOL_ERR_INVALID;
  if (xyzs && !species_idx) return FENNOL_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  FNL_LAUNCH_PDL(k_md_step, (natoms + 255) / 256, 256, 0, st, 
      natoms, dt, x, v, inv_mass, (const float4*)forces4, force_scale, a1, a2, seed, step_counter,
      coords, species_idx, (float4*)xyzs, x_ref, half_skin * half_skin, rebuild_flag);
  FNL_CHECK_LAUNCH();
  if (step_counter) {
    FNL_LAUNCH_PDL(k_inc_counter, 1, 1, 0, st, step_counter);
    FNL_CHECK_LAUNCH();
  }
  return FENNOL_OK;
}

extern "C" int fennol_md_step_systems(int natoms, int nsys, double dt, double* x, double* v,
                                      const double* inv_mass, const float* forces4, double force_scale,
                                      double a1, const double* a2, const int* atom_sys, const int* sys_start,
                                      const unsigned long long* sys_seed, unsigned long long* sys_step,
                                      float* coords, const int* species_idx, float* xyzs,
                                      const double* x_ref, double half_skin, int* rebuild_flag,
                                      void* stream) {
  if (natoms < 0 || nsys < 0 || !(dt > 0)) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!x || !v || !inv_mass || !forces4 || !atom_sys || !sys_start || !sys_seed || !sys_step || nsys == 0)
    return FENNOL_ERR_INVALID;
  if (xyzs && !species_idx) return FENNOL_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  FNL_LAUNCH_PDL(k_md_step_systems, (natoms + 255) / 256, 256, 0, st, 
      natoms, dt, x, v, inv_mass, (const float4*)forces4, force_scale, a1, a2, atom_sys, sys_start, sys_seed,
      sys_step, coords, species_idx, (float4*)xyzs, x_ref, half_skin * half_skin, rebuild_flag);
  FNL_CHECK_LAUNCH();
  FNL_LAUNCH_PDL(k_inc_steps, (nsys + 255) / 256, 256, 0, st, nsys, sys_step);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_md_mark_rebuilt(int natoms, const double* x, double* x_ref, int* rebuild_flag,
                                      void* stream) {
  if (natoms < 0 || !x || !x_ref || !rebuild_flag) return FENNOL_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  if (natoms > 0) {
    FNL_LAUNCH_PDL(k_mark_rebuilt, (3 * natoms + 255) / 256, 256, 0, st, natoms, x, x_ref, rebuild_flag);
    FNL_CHECK_LAUNCH();
  }
  FNL_LAUNCH_PDL(k_clear_flag, 1, 1, 0, st, rebuild_flag);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_md_kinetic(int natoms, const double* v, const double* inv_mass, double* kinetic,
                                 void* stream) {
  if (natoms < 0 || !kinetic) return FENNOL_ERR_INVALID;
  if (natoms > 0 && (!v || !inv_mass)) return FENNOL_ERR_INVALID;
  FNL_LAUNCH_PDL(k_kinetic, 1, 1024, 0, (cudaStream_t)stream, natoms, v, inv_mass, kinetic);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

// ---------------------------------------------------------------------------
// Non-finite check of up to four buffers in one launch.
// ---------------------------------------------------------------------------
namespace {
struct FiniteBufs {
  const void* ptr[4];
  unsigned long long count[4];
  int is_double[4];
  int n;
};

__global__ void k_check_finite(const FiniteBufs b, int* status) {
  pdl_wait();
  bool bad = false;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (int k = 0; k < b.n; ++k) {
    const size_t n = b.count[k];
    if (b.is_double[k]) {
      const double* p = (const double*)b.ptr[k];
      for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) bad |= !isfinite(p[i]);
    } else {
      const float* p = (const float*)b.ptr[k];
      for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) bad |= !isfinite(p[i]);
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status + fnl::ST_NONFINITE, 1);
}
}  // namespace

extern "C" int fennol_check_finite(int nbuf, const void* const* host_ptrs, const size_t* host_counts,
                                   const int* host_is_double, int* status, void* stream) {
  if (nbuf < 0 || nbuf > 4 || !status) return FENNOL_ERR_INVALID;
  if (nbuf > 0 && (!host_ptrs || !host_counts || !host_is_double)) return FENNOL_ERR_INVALID;
  FiniteBufs b{};
  size_t total = 0;
  for (int k = 0; k < nbuf; ++k) {
    if (host_counts[k] > 0 && !host_ptrs[k]) return FENNOL_ERR_INVALID;
    b.ptr[k] = host_ptrs[k];
    b.count[k] = host_counts[k];
    b.is_double[k] = host_is_double[k] != 0;
    total = host_counts[k] > total ? host_counts[k] : total;
  }
  b.n = nbuf;
  if (total == 0) return FENNOL_OK;
  size_t blocks = (total + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  FNL_LAUNCH_PDL(k_check_finite, dim3((unsigned)blocks), dim3(256), 0, (cudaStream_t)stream, b, status);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}
