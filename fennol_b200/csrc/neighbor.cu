// Neighbour search on sm_100a: periodic cell list with warp-ballot compaction,
// an all-pairs path for molecules and small boxes, and the skin/cutoff filter.
//
// Replaces FeNNol's GraphGenerator.__call__/process/update_skin and
// GraphFilter (src/fennol/models/preprocessing.py:74-696, 834-960).  The
// pair predicate reproduces the reference's float32 numpy arithmetic exactly
// (see common.cuh: no FMA contraction, (x*x+y*y)+z*z, threshold rounded from
// the double cutoff), so the kept pair set is the reference's.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"

using namespace fnl;

namespace {

constexpr int kBuildWarps = 4;      // warps per block in the row builders
constexpr int kMaxRow = 1024;       // longest neighbour row accepted

struct SysView {
  const int* start;
  const int* mode;
  const float* cell;
  const float* recip;
  const int* grid;
  const int* nrep;
};

struct GraphWs {
  int* counts;      // [C]
  int* starts;      // [C+1]
  int* cursor;      // [C]
  int* cell_atoms;  // [N]
  int* atom_cell;   // [N]  (-1: all-pairs system)
  float4* pos;      // [N]  wrapped (general PBC) or raw positions
  unsigned* at;     // [N]  packed wrap shift (general PBC)
};

__host__ size_t ws_layout(int n, int c, char* base, GraphWs* w) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = (off + bytes + 255) / 256 * 256;
    return o;
  };
  size_t o_counts = take(sizeof(int) * (size_t)std::max(c, 1));
  size_t o_starts = take(sizeof(int) * (size_t)(c + 1));
  size_t o_cursor = take(sizeof(int) * (size_t)std::max(c, 1));
  size_t o_catoms = take(sizeof(int) * (size_t)std::max(n, 1));
  size_t o_acell = take(sizeof(int) * (size_t)std::max(n, 1));
  size_t o_pos = take(sizeof(float4) * (size_t)std::max(n, 1));
  size_t o_at = take(sizeof(unsigned) * (size_t)std::max(n, 1));
  if (w && base) {
    w->counts = (int*)(base + o_counts);
    w->starts = (int*)(base + o_starts);
    w->cursor = (int*)(base + o_cursor);
    w->cell_atoms = (int*)(base + o_catoms);
    w->atom_cell = (int*)(base + o_acell);
    w->pos = (float4*)(base + o_pos);
    w->at = (unsigned*)(base + o_at);
  }
  return off;
}

// ---------------------------------------------------------------------------
// 1. per atom: arithmetic position (wrapped for general PBC), wrap shift,
//    cell id and cell histogram.
// ---------------------------------------------------------------------------
__global__ void k_prepare(const float* __restrict__ coords, int n, const int* __restrict__ atom_sys,
                          SysView sv, GraphWs w, const int* enable_flag) {
  pdl_wait();
  if (enable_flag && *enable_flag == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = atom_sys[i];
  int mode = sv.mode[b];
  float x = coords[3 * i], y = coords[3 * i + 1], z = coords[3 * i + 2];
  unsigned at = 0;
  const float* c = sv.cell + 9 * b;
  const float* r = sv.recip + 9 * b;
  if (mode == FENNOL_PBC_GENERAL) {
    // at_shifts = -floor(x @ recip); x += at_shifts @ cell  (preprocessing.py:144-158)
    float ax = -floorf(frac_exact(x, y, z, r, 0));
    float ay = -floorf(frac_exact(x, y, z, r, 1));
    float az = -floorf(frac_exact(x, y, z, r, 2));
    add_shift(x, y, z, ax, ay, az, c);
    at = pack_shift((int)ax, (int)ay, (int)az);
  }
  w.pos[i] = make_float4(x, y, z, 0.f);
  w.at[i] = at;
  const int* g = sv.grid + 4 * b;
  if (mode != FENNOL_PBC_NONE && g[0] > 0) {
    int nc[3] = {g[0], g[1], g[2]};
    int ci[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float f = frac_exact(x, y, z, r, d);
      f -= floorf(f);
      int k = (int)(f * (float)nc[d]);
      ci[d] = k < 0 ? 0 : (k >= nc[d] ? nc[d] - 1 : k);
    }
    int cell = g[3] + (ci[0] * nc[1] + ci[1]) * nc[2] + ci[2];
    w.atom_cell[i] = cell;
    atomicAdd(w.counts + cell, 1);
  } else {
    w.atom_cell[i] = -1;
  }
}

// ---------------------------------------------------------------------------
// 2. exclusive scan of the cell histogram (one block), cursor = start.
// ---------------------------------------------------------------------------
__global__ void k_scan(GraphWs w, int c, const int* enable_flag) {
  pdl_wait();
  if (enable_flag && *enable_flag == 0) return;
  __shared__ int warp_sums[32];
  __shared__ int carry;
  int tid = threadIdx.x;
  if (tid == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < c; base += blockDim.x) {
    int idx = base + tid;
    int v = idx < c ? w.counts[idx] : 0;
    int lane = tid & 31, wid = tid >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warp_sums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      int nw = blockDim.x >> 5;
      int s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += t;
      }
      if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    int excl = carry + (wid > 0 ? warp_sums[wid - 1] : 0) + incl - v;
    if (idx < c) {
      w.starts[idx] = excl;
      w.cursor[idx] = excl;
    }
    __syncthreads();
    if (tid == blockDim.x - 1) carry = excl + v;
    __syncthreads();
  }
  if (tid == 0) w.starts[c] = carry;
}

// 3. scatter atoms into their cells (order inside a cell is arbitrary until
//    k_sort_cells puts each cell in increasing index order).
__global__ void k_scatter(int n, GraphWs w, const int* enable_flag) {
  pdl_wait();
  if (enable_flag && *enable_flag == 0) return;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int cell = w.atom_cell[i];
  if (cell < 0) return;
  int slot = atomicAdd(w.cursor + cell, 1);
  w.cell_atoms[slot] = i;
}

// Candidate test for the pair (i, j) with image shift `img` (general PBC) or
// the rounding shift (minimum image); returns true and the stored shift when
// d^2 < rc2.
__device__ __forceinline__ bool pair_test(int mode, float4 pi, float4 pj, unsigned ati, unsigned atj,
                                          int ix, int iy, int iz, const float* c, const float* r,
                                          float rc2, unsigned& shift_out) {
  float vx = __fsub_rn(pj.x, pi.x), vy = __fsub_rn(pj.y, pi.y), vz = __fsub_rn(pj.z, pi.z);
  int sx = 0, sy = 0, sz = 0;
  if (mode == FENNOL_PBC_MINIMUM_IMAGE) {
    // pbc_shifts = -round(vec @ recip); vec += pbc_shifts @ cell (preprocessing.py:127-143)
    float fx = -rintf(frac_exact(vx, vy, vz, r, 0));
    float fy = -rintf(frac_exact(vx, vy, vz, r, 1));
    float fz = -rintf(frac_exact(vx, vy, vz, r, 2));
    add_shift(vx, vy, vz, fx, fy, fz, c);
    sx = (int)fx;
    sy = (int)fy;
    sz = (int)fz;
  } else if (mode == FENNOL_PBC_GENERAL) {
    if (ix | iy | iz) add_shift(vx, vy, vz, (float)ix, (float)iy, (float)iz, c);
    int ax, ay, az, bx, by, bz;
    unpack_shift(ati, ax, ay, az);
    unpack_shift(atj, bx, by, bz);
    sx = ix + bx - ax;
    sy = iy + by - ay;
    sz = iz + bz - az;
  }
  float d2 = dist2_exact(vx, vy, vz);
  shift_out = pack_shift(sx, sy, sz);
  return d2 < rc2;
}

// Append the candidates selected by `keep` (one per lane) to row `base` in
// global memory, in lane order after the `count` entries already there.
__device__ __forceinline__ void row_append(bool keep, int j, unsigned sh, int* __restrict__ nbr_j,
                                           unsigned* __restrict__ nbr_shift, size_t base, int cap, int& count,
                                           int lane) {
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (keep) {
    const int pos = count + warp_exclusive_prefix(m, lane);
    if (pos < cap) {
      nbr_j[base + pos] = j;
      nbr_shift[base + pos] = sh;
    }
  }
  count += __popc(m);
}

__device__ __forceinline__ void row_finish(int i, int count, int cap, int* __restrict__ nbr_count, int* status,
                                           int lane) {
  if (lane == 0) {
    nbr_count[i] = count < cap ? count : cap;
    if (count > cap) status_set(status, ST_NBR_OVERFLOW);
    status_max(status, ST_NBR_MAXCOUNT, count);
  }
}

// ---------------------------------------------------------------------------
// 3b. each cell's atom list in increasing index order (warp per cell), so
//     that rows built in stencil order are deterministic.
// ---------------------------------------------------------------------------
constexpr int kCellSortMax = 512;  // larger cells (densities far above a liquid's) keep scatter order

__global__ void __launch_bounds__(256) k_sort_cells(int c, GraphWs w, const int* enable_flag) {
  pdl_wait();
  if (enable_flag && *enable_flag == 0) return;
  __shared__ int buf[8][kCellSortMax];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cell = blockIdx.x * 8 + warp;
  if (cell >= c) return;
  const int s0 = w.starts[cell], n = w.starts[cell + 1] - s0;
  if (n <= 1) return;
  if (n <= 32) {
    int v = lane < n ? w.cell_atoms[s0 + lane] : 0x7fffffff;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
      for (int j = k >> 1; j > 0; j >>= 1) {
        const int o = __shfl_xor_sync(0xffffffffu, v, j);
        const bool up = (lane & k) == 0, lower = (lane & j) == 0;
        v = (lower == up) ? min(v, o) : max(v, o);
      }
    }
    if (lane < n) w.cell_atoms[s0 + lane] = v;
    return;
  }
  if (n > kCellSortMax) return;
  int m = 64;
  while (m < n) m <<= 1;
  int* b = buf[warp];
  for (int k = lane; k < m; k += 32) b[k] = k < n ? w.cell_atoms[s0 + k] : 0x7fffffff;
  __syncwarp();
  for (int k = 2; k <= m; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int idx = lane; idx < m; idx += 32) {
        const int ixj = idx ^ j;
        if (ixj > idx) {
          const int a = b[idx], bb = b[ixj];
          if ((a > bb) == ((idx & k) == 0)) {
            b[idx] = bb;
            b[ixj] = a;
          }
        }
      }
      __syncwarp();
    }
  }
  for (int k = lane; k < n; k += 32) w.cell_atoms[s0 + k] = b[k];
}

// ---------------------------------------------------------------------------
// 4a. cell-list rows: one warp per atom.  The 27 stencil cells' atom ranges
//     are concatenated, so every 32-lane round tests 32 candidates whatever
//     the cell sizes; kept pairs go straight to the row in candidate order
//     (stencil cell, then atom index), which makes the rows deterministic.
// ---------------------------------------------------------------------------
// Row of atom i from its 27 stencil cells (warp-collective).
__device__ __forceinline__ void cell_row(int i, const int* __restrict__ atom_sys, const SysView& sv,
                                         const GraphWs& w, float rc2, int cap, int* __restrict__ nbr_j,
                                         unsigned* __restrict__ nbr_shift, int* __restrict__ nbr_count,
                                         int* status, int lane) {
  const int cell = w.atom_cell[i];
  if (cell < 0) return;  // all-pairs system
  const int b = atom_sys[i];
  const int mode = sv.mode[b];
  const float* c = sv.cell + 9 * b;
  const float* r = sv.recip + 9 * b;
  const int* g = sv.grid + 4 * b;
  const int nx = g[0], ny = g[1], nz = g[2], off = g[3];
  const int local = cell - off;
  const int cz = local % nz, cy = (local / nz) % ny, cx = local / (ny * nz);
  // lane s < 27: stencil cell s = (dx, dy, dz) + 1 in base 3, its atom range and wrap
  int s0 = 0, cnt = 0, wrap = 0;
  if (lane < 27) {
    int ex = cx + lane / 9 - 1, ey = cy + (lane / 3) % 3 - 1, ez = cz + lane % 3 - 1;
    int wx = 0, wy = 0, wz = 0;
    if (ex < 0) { ex += nx; wx = -1; } else if (ex >= nx) { ex -= nx; wx = 1; }
    if (ey < 0) { ey += ny; wy = -1; } else if (ey >= ny) { ey -= ny; wy = 1; }
    if (ez < 0) { ez += nz; wz = -1; } else if (ez >= nz) { ez -= nz; wz = 1; }
    const int nc = off + (ex * ny + ey) * nz + ez;
    s0 = w.starts[nc];
    cnt = w.starts[nc + 1] - s0;
    wrap = (wx + 1) | ((wy + 1) << 2) | ((wz + 1) << 4);
  }
  int incl = cnt;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  const int first = incl - cnt;  // first candidate of stencil cell `lane`
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  const float4 pi = w.pos[i];
  const unsigned ati = w.at[i];
  const size_t base = (size_t)i * cap;
  int count = 0;
  for (int k0 = 0; k0 < total; k0 += 32) {
    const int k = k0 + lane;
    // stencil cell of candidate k: the last s < 27 with first[s] <= k
    int sc = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const int cand = sc + step;
      const int fc = __shfl_sync(0xffffffffu, first, cand & 31);
      if (cand < 27 && fc <= k) sc = cand;
    }
    const int sfirst = __shfl_sync(0xffffffffu, first, sc);
    const int sstart = __shfl_sync(0xffffffffu, s0, sc);
    const int swrap = __shfl_sync(0xffffffffu, wrap, sc);
    bool keep = false;
    int j = -1;
    unsigned sh = 0;
    if (k < total) {
      j = w.cell_atoms[sstart + k - sfirst];
      if (j != i)
        keep = pair_test(mode, pi, w.pos[j], ati, w.at[j], (swrap & 3) - 1, ((swrap >> 2) & 3) - 1,
                         ((swrap >> 4) & 3) - 1, c, r, rc2, sh);
    }
    row_append(keep, j, sh, nbr_j, nbr_shift, base, cap, count, lane);
  }
  row_finish(i, count, cap, nbr_count, status, lane);
}

// ---------------------------------------------------------------------------
// 4a'. cell-list rows with the stencil staged in shared memory: one block per
//      cell gathers the candidates of its 27 stencil cells (position, index,
//      wrap shift, stencil cell) once, and its warps build the rows of the
//      cell's atoms from that copy; every candidate is read from global memory
//      once per cell instead of once per atom.  Candidates are kept in the
//      order of 4a (stencil cell, then atom index), so the rows are the same.
//      A cell whose stencil holds more than kStageCand candidates falls back
//      to the per-atom gathers of 4a.
// ---------------------------------------------------------------------------
constexpr int kStageCand = 1024;
constexpr int kCellWarps = 8;  // warps per cell block: the atoms of a cell (~14-24 in a liquid) are shared out

// Position moved into the box by whole cell vectors, -floor of its fractional
// coordinates as the binning takes them (k_prepare).
__device__ __forceinline__ float4 wrapped(float4 p, const float* c, const float* r) {
  float x = p.x, y = p.y, z = p.z;
  const float ax = -floorf(frac_exact(x, y, z, r, 0));
  const float ay = -floorf(frac_exact(x, y, z, r, 1));
  const float az = -floorf(frac_exact(x, y, z, r, 2));
  add_shift(x, y, z, ax, ay, az, c);
  return make_float4(x, y, z, 0.f);
}

__global__ void __launch_bounds__(kCellWarps * 32)
k_build_cells_staged(int ncells, const int* __restrict__ atom_sys, SysView sv, GraphWs w, float rc2, int cap,
                     int* __restrict__ nbr_j, unsigned* __restrict__ nbr_shift, int* __restrict__ nbr_count,
                     int* status, const int* enable_flag) {
  pdl_wait();
  if (enable_flag && *enable_flag == 0) return;
  __shared__ float4 c_pos[kStageCand];
  __shared__ float4 c_posw[kStageCand];  // minimum image: positions wrapped into the box (pre-test)
  __shared__ int c_j[kStageCand];
  __shared__ unsigned c_at[kStageCand];
  __shared__ unsigned char c_sc[kStageCand];
  __shared__ int s_first[28], s_start[27], s_wrap[27];
  __shared__ float4 s_shift[27];               // wrap @ cell of each stencil cell
  __shared__ int s_queue[kCellWarps][64];     // per warp: candidates that passed the pre-test
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const unsigned lt = (1u << lane) - 1u;
  // pre-test threshold: a little above rc^2, far beyond the rounding difference
  // between the pre-test's distance and the exact one
  const float rc_pre = sqrtf(rc2) + 0.05f, rc2_pre = rc_pre * rc_pre;
  for (int cell = blockIdx.x; cell < ncells; cell += gridDim.x) {
    const int a0 = w.starts[cell], na = w.starts[cell + 1] - a0;
    if (na == 0) continue;  // block-uniform
    const int b = atom_sys[w.cell_atoms[a0]];
    const int mode = sv.mode[b];
    const float* c = sv.cell + 9 * b;
    const float* r = sv.recip + 9 * b;
    const int* g = sv.grid + 4 * b;
    const int nx = g[0], ny = g[1], nz = g[2], off = g[3];
    const int local = cell - off;
    const int cz = local % nz, cy = (local / nz) % ny, cx = local / (ny * nz);
    if (warp == 0) {
      int s0 = 0, cnt = 0, wrap = 0;
      if (lane < 27) {
        int ex = cx + lane / 9 - 1, ey = cy + (lane / 3) % 3 - 1, ez = cz + lane % 3 - 1;
        int wx = 0, wy = 0, wz = 0;
        if (ex < 0) { ex += nx; wx = -1; } else if (ex >= nx) { ex -= nx; wx = 1; }
        if (ey < 0) { ey += ny; wy = -1; } else if (ey >= ny) { ey -= ny; wy = 1; }
        if (ez < 0) { ez += nz; wz = -1; } else if (ez >= nz) { ez -= nz; wz = 1; }
        const int nc = off + (ex * ny + ey) * nz + ez;
        s0 = w.starts[nc];
        cnt = w.starts[nc + 1] - s0;
        wrap = (wx + 1) | ((wy + 1) << 2) | ((wz + 1) << 4);
      }
      int incl = cnt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane < 27) {
        s_first[lane] = incl - cnt;
        s_start[lane] = s0;
        s_wrap[lane] = wrap;
        const float wx = (float)((wrap & 3) - 1), wy = (float)(((wrap >> 2) & 3) - 1),
                    wz = (float)(((wrap >> 4) & 3) - 1);
        s_shift[lane] = make_float4(wx * c[0] + wy * c[3] + wz * c[6], wx * c[1] + wy * c[4] + wz * c[7],
                                    wx * c[2] + wy * c[5] + wz * c[8], 0.f);
      }
      if (lane == 26) s_first[27] = incl;
    }
    __syncthreads();
    const int total = s_first[27];
    if (total <= kStageCand) {
      for (int k = tid; k < total; k += kCellWarps * 32) {
        // stencil cell of candidate k: the last s < 27 with s_first[s] <= k
        int sc = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1)
          if (sc + step < 27 && s_first[sc + step] <= k) sc += step;
        const int j = w.cell_atoms[s_start[sc] + k - s_first[sc]];
        const float4 pj = w.pos[j];
        c_pos[k] = pj;
        if (mode == FENNOL_PBC_MINIMUM_IMAGE) c_posw[k] = wrapped(pj, c, r);
        c_j[k] = j;
        c_at[k] = w.at[j];
        c_sc[k] = (unsigned char)sc;
      }
      __syncthreads();
      int* q = s_queue[warp];
      for (int a = warp; a < na; a += kCellWarps) {
        const int i = w.cell_atoms[a0 + a];
        const float4 pi = w.pos[i];
        const unsigned ati = w.at[i];
        const size_t base = (size_t)i * cap;
        int count = 0;
        if (mode == FENNOL_PBC_MINIMUM_IMAGE) {
          // A candidate within the cutoff in the reference's minimum image lies
          // in an adjacent cell, so that image is the box-wrapped positions
          // plus the stencil cell's wrap: a cheap distance in that image (any
          // rounding; 0.05 A of margin) rejects the far candidates, and the
          // survivors, queued in candidate order, take the exact test 32 at a
          // time.  The rows are those of the exact test alone.
          const float4 piw = wrapped(pi, c, r);
          auto exact_round = [&](int nq) {
            const int kk = lane < nq ? q[lane] : -1;
            bool keep = false;
            int j = -1;
            unsigned sh = 0;
            if (kk >= 0) {
              j = c_j[kk];
              keep = pair_test(mode, pi, c_pos[kk], ati, c_at[kk], 0, 0, 0, c, r, rc2, sh);
            }
            row_append(keep, j, sh, nbr_j, nbr_shift, base, cap, count, lane);
          };
          int nq = 0;
          for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + lane;
            bool pass = false;
            if (k < total && c_j[k] != i) {
              const float4 pj = c_posw[k], sv4 = s_shift[c_sc[k]];
              const float vx = (pj.x - piw.x) + sv4.x, vy = (pj.y - piw.y) + sv4.y, vz = (pj.z - piw.z) + sv4.z;
              pass = vx * vx + vy * vy + vz * vz < rc2_pre;
            }
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) q[nq + __popc(m & lt)] = k;
            nq += __popc(m);
            __syncwarp();
            if (nq >= 32) {
              exact_round(32);
              const int rest = lane < nq - 32 ? q[32 + lane] : 0;
              __syncwarp();
              if (lane < nq - 32) q[lane] = rest;
              nq -= 32;
              __syncwarp();
            }
          }
          if (nq > 0) exact_round(nq);
        } else {
          for (int k0 = 0; k0 < total; k0 += 32) {
            const int k = k0 + lane;
            bool keep = false;
            int j = -1;
            unsigned sh = 0;
            if (k < total) {
              j = c_j[k];
              if (j != i) {
                const int swrap = s_wrap[c_sc[k]];
                keep = pair_test(mode, pi, c_pos[k], ati, c_at[k], (swrap & 3) - 1, ((swrap >> 2) & 3) - 1,
                                 ((swrap >> 4) & 3) - 1, c, r, rc2, sh);
              }
            }
            row_append(keep, j, sh, nbr_j, nbr_shift, base, cap, count, lane);
          }
        }
        row_finish(i, count, cap, nbr_count, status, lane);
        __syncwarp();  // the queue is reused by the warp's next atom
      }
    } else {
      for (int a = warp; a < na; a += kCellWarps)
        cell_row(w.cell_atoms[a0 + a], atom_sys, sv, w, rc2, cap, nbr_j, nbr_shift, nbr_count, status, lane);
    }
    __syncthreads();  // the stencil tables and candidates are reused by the next cell
  }
}

// ---------------------------------------------------------------------------
// 4b. all-pairs rows (molecules, boxes too small for a 3x3x3 cell stencil).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void allpairs_row(int i, const int* __restrict__ atom_sys, const SysView& sv,
                                             const GraphWs& w, float rc2, int cap, int* __restrict__ nbr_j,
                                             unsigned* __restrict__ nbr_shift, int* __restrict__ nbr_count,
                                             int* status, int lane) {
  if (w.atom_cell[i] >= 0) return;  // cell-list system
  const size_t base = (size_t)i * cap;
  int b = atom_sys[i];
  int mode = sv.mode[b];
  const float* c = sv.cell + 9 * b;
  const float* r = sv.recip + 9 * b;
  int j0 = sv.start[b], j1 = sv.start[b + 1];
  int rx = 0, ry = 0, rz = 0;
  if (mode == FENNOL_PBC_GENERAL) {
    rx = sv.nrep[3 * b];
    ry = sv.nrep[3 * b + 1];
    rz = sv.nrep[3 * b + 2];
  }
  float4 pi = w.pos[i];
  unsigned ati = w.at[i];
  int count = 0;
  for (int ix = -rx; ix <= rx; ++ix)
    for (int iy = -ry; iy <= ry; ++iy)
      for (int iz = -rz; iz <= rz; ++iz) {
        for (int k0 = j0; k0 < j1; k0 += 32) {
          int j = k0 + lane;
          bool keep = false;
          unsigned sh = 0;
          if (j < j1 && j != i)
            keep = pair_test(mode, pi, w.pos[j], ati, w.at[j], ix, iy, iz, c, r, rc2, sh);
          row_append(keep, j, sh, nbr_j, nbr_shift, base, cap, count, lane);
        }
      }
  row_finish(i, count, cap, nbr_count, status, lane);
}

// Also counts the rebuild (one per enabled build) in the status words.
__global__ void __launch_bounds__(kBuildWarps * 32)
k_build_allpairs(int n, const int* __restrict__ atom_sys, SysView sv, GraphWs w, float rc2, int cap,
                 int* __restrict__ nbr_j, unsigned* __restrict__ nbr_shift, int* __restrict__ nbr_count,
                 int* status, const int* enable_flag) {
  pdl_wait();
  if (enable_flag && *enable_flag == 0) return;
  if (status && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(status + ST_REBUILD_COUNT, 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = blockIdx.x * kBuildWarps + warp; i < n; i += gridDim.x * kBuildWarps)
    allpairs_row(i, atom_sys, sv, w, rc2, cap, nbr_j, nbr_shift, nbr_count, status, lane);
}


// ---------------------------------------------------------------------------
// Filter a list to a smaller cutoff (update_skin / GraphFilter).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_filter(const float* __restrict__ coords, int n, const int* __restrict__ atom_sys,
         const float* __restrict__ sys_cell, const int* __restrict__ in_j,
         const unsigned* __restrict__ in_shift, const int* __restrict__ in_count, int in_cap,
         float rc2, int out_cap, int* __restrict__ out_j, unsigned* __restrict__ out_shift,
         int* __restrict__ out_count, int* status) {
  pdl_wait();
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= n) return;
  int i = warp;
  int b = atom_sys[i];
  const float* c = sys_cell ? sys_cell + 9 * b : nullptr;
  float xi = coords[3 * i], yi = coords[3 * i + 1], zi = coords[3 * i + 2];
  int cnt = in_count[i];
  if (cnt > in_cap) cnt = in_cap;
  size_t ib = (size_t)i * in_cap, ob = (size_t)i * out_cap;
  int count = 0;
  // up to kFilterRounds 32-entry rounds at a time: all their index and
  // position loads are in flight together, then the tests and the ordered
  // ballot compaction run round by round (same rows as one round at a time)
  constexpr int kFilterRounds = 4;
  for (int k0 = 0; k0 < cnt; k0 += 32 * kFilterRounds) {
    int j[kFilterRounds];
    unsigned sh[kFilterRounds];
#pragma unroll
    for (int u = 0; u < kFilterRounds; ++u) {
      const int k = k0 + 32 * u + lane;
      j[u] = k < cnt ? in_j[ib + k] : -1;
      sh[u] = k < cnt ? in_shift[ib + k] : 0u;
    }
    float px[kFilterRounds], py[kFilterRounds], pz[kFilterRounds];
#pragma unroll
    for (int u = 0; u < kFilterRounds; ++u) {
      const int jj = j[u] < 0 ? i : j[u];
      px[u] = coords[3 * jj];
      py[u] = coords[3 * jj + 1];
      pz[u] = coords[3 * jj + 2];
    }
#pragma unroll
    for (int u = 0; u < kFilterRounds; ++u) {
      bool keep = false;
      if (j[u] >= 0) {
        float vx = __fsub_rn(px[u], xi);
        float vy = __fsub_rn(py[u], yi);
        float vz = __fsub_rn(pz[u], zi);
        if (sh[u] && c) {
          int sx, sy, sz;
          unpack_shift(sh[u], sx, sy, sz);
          add_shift(vx, vy, vz, (float)sx, (float)sy, (float)sz, c);
        }
        keep = dist2_exact(vx, vy, vz) < rc2;
      }
      unsigned m = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        int pos = count + warp_exclusive_prefix(m, lane);
        if (pos < out_cap) {
          out_j[ob + pos] = j[u];
          out_shift[ob + pos] = sh[u];
        }
      }
      count += __popc(m);
    }
  }
  if (lane == 0) {
    out_count[i] = count < out_cap ? count : out_cap;
    if (count > out_cap) status_set(status, ST_FILTER_OVERFLOW);
    status_max(status, ST_FILTER_MAXCOUNT, count);
  }
}

}  // namespace

extern "C" int fennol_graph_plan(int nsys, const int* host_mode, const float* host_recip,
                                 double cutoff, int* host_grid, int* host_nrep) {
  if (nsys < 0 || !host_mode || !host_grid || !host_nrep || !(cutoff > 0)) return FENNOL_ERR_INVALID;
  long long total = 0;
  for (int b = 0; b < nsys; ++b) {
    int* g = host_grid + 4 * b;
    int* nr = host_nrep + 3 * b;
    g[0] = g[1] = g[2] = 0;
    g[3] = (int)total;
    nr[0] = nr[1] = nr[2] = 0;
    if (host_mode[b] == FENNOL_PBC_NONE) continue;
    if (!host_recip) return FENNOL_ERR_INVALID;
    const float* r = host_recip + 9 * b;
    int nc[3];
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      // |recip column d| as in preprocessing.py:161-163 (float32)
      float s = 0.f;
      for (int k = 0; k < 3; ++k) s += r[3 * k + d] * r[3 * k + d];
      float inv = sqrtf(s);
      nr[d] = (int)std::ceil((float)cutoff * inv);
      // bins wider than the cutoff by a relative margin (binning round-off)
      double width = 1.0 / ((double)inv * cutoff * (1.0 + 1e-5));
      long long k = (long long)std::floor(width);
      if (k > 256) k = 256;
      nc[d] = (int)k;
      if (k < 3) ok = false;
    }
    if (ok) {
      g[0] = nc[0];
      g[1] = nc[1];
      g[2] = nc[2];
      total += (long long)nc[0] * nc[1] * nc[2];
      if (total > (1ll << 30)) return FENNOL_ERR_UNSUPPORTED;
    }
  }
  return (int)total;
}

extern "C" size_t fennol_graph_workspace_bytes(int natoms, int ncells_total) {
  if (natoms < 0 || ncells_total < 0) return 0;
  return ws_layout(natoms, ncells_total, nullptr, nullptr);
}


extern "C" int fennol_graph_build(const float* coords, int natoms, const int* atom_sys, int nsys,
                                  const int* sys_start, const int* sys_mode, const float* sys_cell,
                                  const float* sys_recip, const int* sys_grid, const int* sys_nrep,
                                  int ncells_total, double cutoff, int capacity, int* nbr_j,
                                  unsigned* nbr_shift, int* nbr_count, int* status, void* workspace,
                                  size_t workspace_bytes, const int* enable_flag, void* stream) {
  if (natoms < 0 || nsys <= 0 || capacity <= 0 || capacity > kMaxRow || !(cutoff > 0))
    return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!coords || !atom_sys || !sys_start || !sys_mode || !sys_grid || !sys_nrep || !nbr_j ||
      !nbr_shift || !nbr_count || !workspace || !sys_cell || !sys_recip)
    return FENNOL_ERR_INVALID;
  if (workspace_bytes < fennol_graph_workspace_bytes(natoms, ncells_total)) return FENNOL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  GraphWs w;
  ws_layout(natoms, ncells_total, (char*)workspace, &w);
  SysView sv{sys_start, sys_mode, sys_cell, sys_recip, sys_grid, sys_nrep};
  float rc2 = (float)(cutoff * cutoff);
  if (ncells_total > 0) {
    if (cudaMemsetAsync(w.counts, 0, sizeof(int) * (size_t)ncells_total, st) != cudaSuccess)
      return FENNOL_ERR_CUDA;
  }
  int tb = 256;
  int gb = (natoms + tb - 1) / tb;
  FNL_LAUNCH_PDL(k_prepare, gb, tb, 0, st, coords, natoms, atom_sys, sv, w, enable_flag);
  FNL_CHECK_LAUNCH();
  if (ncells_total > 0) {
    FNL_LAUNCH_PDL(k_scan, 1, 1024, 0, st, w, ncells_total, enable_flag);
    FNL_CHECK_LAUNCH();
    FNL_LAUNCH_PDL(k_scatter, gb, tb, 0, st, natoms, w, enable_flag);
    FNL_CHECK_LAUNCH();
    FNL_LAUNCH_PDL(k_sort_cells, (ncells_total + 7) / 8, 256, 0, st, ncells_total, w, enable_flag);
    FNL_CHECK_LAUNCH();
  }
  // grid-stride row builders: a capped grid keeps the launch cheap when the
  // enable flag turns the build into a no-op
  int gw = std::min((natoms + kBuildWarps - 1) / kBuildWarps, 148 * 16);
  if (ncells_total > 0) {
    const int gc = std::min(ncells_total, 148 * 16);
    FNL_LAUNCH_PDL(k_build_cells_staged, gc, kCellWarps * 32, 0, st, ncells_total, atom_sys, sv, w, rc2, capacity,
                   nbr_j, nbr_shift, nbr_count, status, enable_flag);
    FNL_CHECK_LAUNCH();
  }
  FNL_LAUNCH_PDL(k_build_allpairs, gw, kBuildWarps * 32, 0, st, natoms, atom_sys, sv, w, rc2, capacity, nbr_j, nbr_shift,
                                                     nbr_count, status, enable_flag);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

extern "C" int fennol_graph_filter(const float* coords, int natoms, const int* atom_sys,
                                   const float* sys_cell, const int* in_j, const unsigned* in_shift,
                                   const int* in_count, int in_capacity, double cutoff,
                                   int out_capacity, int* out_j, unsigned* out_shift, int* out_count,
                                   int* status, void* stream) {
  if (natoms < 0 || in_capacity <= 0 || out_capacity <= 0 || !(cutoff > 0)) return FENNOL_ERR_INVALID;
  if (natoms == 0) return FENNOL_OK;
  if (!coords || !atom_sys || !in_j || !in_shift || !in_count || !out_j || !out_shift || !out_count)
    return FENNOL_ERR_INVALID;
  float rc2 = (float)(cutoff * cutoff);
  int threads = 256;
  long long blocks = ((long long)natoms * 32 + threads - 1) / threads;
  FNL_LAUNCH_PDL(k_filter, (unsigned)blocks, threads, 0, (cudaStream_t)stream, 
      coords, natoms, atom_sys, sys_cell, in_j, in_shift, in_count, in_capacity, rc2, out_capacity,
      out_j, out_shift, out_count, status);
  FNL_CHECK_LAUNCH();
  return FENNOL_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of fennol_graph_build.
//
// Callers that cannot allocate device memory -- an XLA FFI handler, where the
// framework owns every buffer and a call must not create memory behind the
// allocator's back, or a stream being captured into a CUDA graph, where
// cudaMalloc is not allowed -- use this entry point.  Its cell-list scratch
// is a file-scope __device__ array sized for at most kStaticMaxAtoms atoms and
// kStaticMaxCells cells; every GPU that loads the library holds that array
// (about 2.2 MB) until the process exits.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr int kStaticMaxAtoms = 65536;
constexpr int kStaticMaxCells = 32768;
constexpr int kStaticMaxDevices = 64;

constexpr size_t round256(size_t v) { return (v + 255) / 256 * 256; }
// Same carve-up as ws_layout(): counts, starts, cursor, cell_atoms, atom_cell, pos, at.
constexpr size_t static_scratch_bytes(size_t n, size_t c) {
  return round256(4 * c) + round256(4 * (c + 1)) + round256(4 * c) + round256(4 * n) + round256(4 * n) +
         round256(16 * n) + round256(4 * n);
}
constexpr size_t kStaticScratchBytes = static_scratch_bytes(kStaticMaxAtoms, kStaticMaxCells);

static __device__ __align__(256) unsigned char g_graph_scratch[kStaticScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kStaticMaxDevices] = {};
unsigned long long g_scratch_ctx[kStaticMaxDevices] = {};

// Unique id of the calling thread's current context (0 if none or if the
// driver lacks cuCtxGetId): a context destroyed and created again, as by
// cudaDeviceReset, has a new id, and device addresses of the old one are void.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(p);
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(p);
  }
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, &id) == 0) return id;
  return 0;
}

// Device address of g_graph_scratch on the current device, looked up once
// per device and context (a new context, e.g. after cudaDeviceReset, is
// looked up again).  In host code the symbol itself is only a host-side
// stand-in.
int scratch_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kStaticMaxDevices) return FENNOL_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  const unsigned long long ctx = current_context_id();
  if (!g_scratch_addr[dev] || ctx != g_scratch_ctx[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_graph_scratch) != cudaSuccess || !p) return FENNOL_ERR_CUDA;
    g_scratch_addr[dev] = p;
    g_scratch_ctx[dev] = current_context_id();  // the lookup may have created the context
  }
  *out = g_scratch_addr[dev];
  return FENNOL_OK;
}

}  // namespace

extern "C" int fennol_graph_build_noalloc(const float* coords, int natoms, const int* atom_sys, int nsys,
                                          const int* sys_start, const int* sys_mode, const float* sys_cell,
                                          const float* sys_recip, const int* sys_grid, const int* sys_nrep,
                                          int ncells_total, double cutoff, int capacity, int* nbr_j,
                                          unsigned* nbr_shift, int* nbr_count, int* status,
                                          const int* enable_flag, void* stream) {
  if (natoms > kStaticMaxAtoms || ncells_total > kStaticMaxCells) return FENNOL_ERR_STATIC_LIMIT;
  if (natoms < 0 || ncells_total < 0) return FENNOL_ERR_INVALID;
  if (fennol_graph_workspace_bytes(natoms, ncells_total) > kStaticScratchBytes) return FENNOL_ERR_STATIC_LIMIT;
  void* scratch = nullptr;
  int rc = scratch_address(&scratch);
  if (rc != FENNOL_OK) return rc;
  // fennol_graph_build clears the cell histogram it needs before use; the
  // rest of the scratch is fully rewritten by each call.
  return fennol_graph_build(coords, natoms, atom_sys, nsys, sys_start, sys_mode, sys_cell, sys_recip,
                            sys_grid, sys_nrep, ncells_total, cutoff, capacity, nbr_j, nbr_shift, nbr_count,
                            status, scratch, kStaticScratchBytes, enable_flag, stream);
}

extern "C" int fennol_graph_noalloc_limits(int* max_atoms, int* max_cells, size_t* scratch_bytes) {
  if (max_atoms) *max_atoms = kStaticMaxAtoms;
  if (max_cells) *max_cells = kStaticMaxCells;
  if (scratch_bytes) *scratch_bytes = kStaticScratchBytes;
  return FENNOL_OK;
}
