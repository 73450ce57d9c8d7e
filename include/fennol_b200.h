/*
 * fennol_b200 -- C ABI of the B200 (sm_100a) energy-and-force path of an
 * ANI-2x-style potential.
 *
 * Conventions shared by every entry point:
 *   - all array pointers are DEVICE pointers unless the name says host_;
 *   - the library allocates nothing: the caller passes every output and
 *     workspace buffer (sizes come from the *_bytes queries);
 *   - `stream` is a cudaStream_t passed as void*; every launch is enqueued
 *     on it and nothing synchronises the device;
 *   - return value: FENNOL_OK (0) or a negative FENNOL_ERR_* code; nothing
 *     aborts and nothing throws.  Capacity problems found on the device are
 *     reported through the int32 `status` words (see FENNOL_ST_*), like the
 *     reference's `overflow` flags, and the caller regrows and relaunches;
 *   - atoms of one system are contiguous; `atom_sys[i]` is FeNNol's
 *     `batch_index`, `sys_start[b]` the first atom of system b;
 *   - cells are row-major 3x3, rows are lattice vectors (FeNNol `cells[b]`);
 *     a periodic image of atom j is x_j + shift @ cell.
 *
 * Reference interfaces named below are files of thomasple/FeNNol.
 */
#ifndef FENNOL_B200_H
#define FENNOL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FENNOL_OK 0
#define FENNOL_ERR_INVALID (-1)
#define FENNOL_ERR_CUDA (-2)
#define FENNOL_ERR_UNSUPPORTED (-3)
#define FENNOL_ERR_WORKSPACE (-4)
#define FENNOL_ERR_STATIC_LIMIT (-5) /* input larger than a fixed in-library scratch */

#define FENNOL_STATUS_WORDS 9
#define FENNOL_ST_NBR_OVERFLOW 0
#define FENNOL_ST_NBR_MAXCOUNT 1
#define FENNOL_ST_FILTER_OVERFLOW 2
#define FENNOL_ST_FILTER_MAXCOUNT 3
#define FENNOL_ST_ANG_OVERFLOW 4
#define FENNOL_ST_ANG_MAXCOUNT 5
#define FENNOL_ST_CELL_OVERFLOW 6
#define FENNOL_ST_REBUILD_COUNT 7
#define FENNOL_ST_NONFINITE 8        /* a checked buffer held a NaN or an infinity */

/* Periodic handling of one system (GraphGenerator, preprocessing.py:117-258). */
#define FENNOL_PBC_NONE 0
#define FENNOL_PBC_MINIMUM_IMAGE 1
#define FENNOL_PBC_GENERAL 2

/* Angular neighbours per centre atom that the AEV kernels stage on chip:
 * the capacity of the radial rows they read, at most this value.  A centre
 * has no more angular than radial neighbours, so rows of capacity up to 256
 * never overflow it; longer rows report FENNOL_ST_ANG_OVERFLOW beyond 256. */
#define FENNOL_MAX_ANGULAR_NEIGHBORS 256

/* ------------------------------------------------------------------------ */
/* Library                                                                   */
/* ------------------------------------------------------------------------ */

/* Version string of the build. */
const char* fennol_version(void);

/* ------------------------------------------------------------------------ */
/* Neighbour search                                                          */
/* ------------------------------------------------------------------------ */

/*
 * Host-only planning of the cell grid for each system.  Replaces the shape
 * bookkeeping of GraphGenerator.__call__ (preprocessing.py:90-100, 168-182):
 * for periodic systems whose cell holds at least 3 bins of width > cutoff
 * along every axis the builder uses a cell list, otherwise it tests all pairs
 * (with image repeats ceil(cutoff*|recip column|) for general PBC).
 *   host_mode[nsys], host_recip[nsys*9]: inputs;
 *   host_grid[nsys*4] out: (nx, ny, nz, first global cell) or zeros;
 *   host_nrep[nsys*3] out: image repeats for all-pairs general PBC;
 *   returns the total number of cells (>= 0) or a negative error.
 */
int fennol_graph_plan(int nsys, const int* host_mode, const float* host_recip, double cutoff,
                      int* host_grid, int* host_nrep);

/* Workspace of fennol_graph_build, in bytes. */
size_t fennol_graph_workspace_bytes(int natoms, int ncells_total);

/*
 * Periodic cell-list neighbour search.  Replaces GraphGenerator.__call__ and
 * GraphGenerator.process (preprocessing.py:74-355, 369-638).
 *
 * For every atom i it writes the row of all j != i of the same system (and
 * periodic image) with d^2 < cutoff^2, where d^2 is computed exactly like the
 * reference's float32 numpy path: vec = x_j - x_i, minimum image
 * s = -rint(vec @ recip), vec += s @ cell, d^2 = (x*x + y*y) + z*z, compared
 * with (float)(cutoff*cutoff) (cutoff is passed in double precision so the
 * threshold rounds exactly like the reference's Python float).  General PBC wraps atoms with -floor(x @ recip)
 * first and stores shift = image + at_shift[j] - at_shift[i] (:340-346).
 * A row lists its pairs in a fixed order (cell-list systems: stencil cell,
 * then increasing j; all-pairs systems: image, then increasing j), so the
 * result is deterministic and independent of the other systems in the batch.
 * Outputs: nbr_j[natoms*capacity], nbr_shift[natoms*capacity] (packed
 * signed bytes x | y<<8 | z<<16), nbr_count[natoms] (clamped to capacity).
 * Overflow sets status[FENNOL_ST_NBR_OVERFLOW] and the needed row length goes
 * to status[FENNOL_ST_NBR_MAXCOUNT] (the reference's check_reallocate,
 * preprocessing.py:357-367).  If `enable_flag` is not NULL the launch does
 * nothing unless *enable_flag != 0 (device-side rebuild trigger); on a
 * rebuild it increments status[FENNOL_ST_REBUILD_COUNT].
 */
int fennol_graph_build(const float* coords, int natoms, const int* atom_sys, int nsys,
                       const int* sys_start, const int* sys_mode, const float* sys_cell,
                       const float* sys_recip, const int* sys_grid, const int* sys_nrep,
                       int ncells_total, double cutoff, int capacity, int* nbr_j,
                       unsigned* nbr_shift, int* nbr_count, int* status, void* workspace,
                       size_t workspace_bytes, const int* enable_flag, void* stream);

/*
 * Allocation-free variant of fennol_graph_build (no counterpart in the
 * reference).  For callers that cannot allocate device memory: an XLA FFI
 * handler, where the framework owns every buffer, or a stream under CUDA
 * graph capture, where cudaMalloc is not allowed.  Same arguments and
 * results as fennol_graph_build, but the cell-list scratch is a fixed array
 * inside the library (one per GPU, about 2.2 MB, held until the process
 * exits) instead of a caller workspace; the caller still passes inputs and
 * outputs.  Limits: natoms <= 65536 and ncells_total <= 32768, otherwise
 * FENNOL_ERR_STATIC_LIMIT and nothing is launched (see
 * fennol_graph_noalloc_limits).  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress); make that first call
 * before any stream capture.  The address is kept per device and context:
 * after cudaDeviceReset (a new context) the next call looks it up again, so
 * make that call outside stream capture too.  All calls share the one array: calls whose
 * work overlaps on the GPU (two streams, or two threads) race on it and must
 * be serialised by the caller.  Allocates nothing.
 */
int fennol_graph_build_noalloc(const float* coords, int natoms, const int* atom_sys, int nsys,
                               const int* sys_start, const int* sys_mode, const float* sys_cell,
                               const float* sys_recip, const int* sys_grid, const int* sys_nrep,
                               int ncells_total, double cutoff, int capacity, int* nbr_j,
                               unsigned* nbr_shift, int* nbr_count, int* status,
                               const int* enable_flag, void* stream);

/* Limits and scratch size of fennol_graph_build_noalloc (host only). */
int fennol_graph_noalloc_limits(int* max_atoms, int* max_cells, size_t* scratch_bytes);

/*
 * Re-filter a neighbour list to a smaller cutoff from current positions.
 * Replaces GraphGenerator.update_skin (preprocessing.py:640-696) when applied
 * to the skin list, and GraphFilter (preprocessing.py:834-960) when applied
 * to the radial list with the angular cutoff.  vec = (x_j - x_i) + s @ cell
 * with the same float32 arithmetic; kept rows preserve the input order.
 */
int fennol_graph_filter(const float* coords, int natoms, const int* atom_sys,
                        const float* sys_cell, const int* in_j, const unsigned* in_shift,
                        const int* in_count, int in_capacity, double cutoff, int out_capacity,
                        int* out_j, unsigned* out_shift, int* out_count, int* status,
                        void* stream);

/* ------------------------------------------------------------------------ */
/* ANI atomic environment vectors                                            */
/* ------------------------------------------------------------------------ */

/* Hyper-parameters of ANIAEV (embeddings/ani.py:18-44). */
typedef struct fennol_aev_params {
  int num_species;          /* S <= 8 */
  int radial_divisions;     /* 16 or 32 */
  int angular_divisions;    /* angular_dist_divisions */
  int angle_sections;       /* angular_divisions * angle_sections == 32 */
  double radial_cutoff;
  double angular_cutoff;
  float radial_eta;
  float angular_eta;
  float zeta;
  float radial_start;
  float angular_start;
} fennol_aev_params;

/* AEV width S*RD + S(S+1)/2*AD*AS, or -1 for unsupported parameters. */
int fennol_aev_length(const fennol_aev_params* p);

/*
 * Host only.  The 64-column chunks of an AEV row (layout of
 * fennol_aev_forward) that can be non-zero when the atoms' species indices
 * all lie in species_mask (bit s = species s present): the radial blocks of
 * the present species and the angular blocks of their pairs.  Bit c of the
 * result covers columns [64c, 64c + 64); widths beyond 64 chunks are not
 * representable (0 is returned, as for unsupported parameters).
 */
unsigned long long fennol_aev_active_chunks(const fennol_aev_params* p, unsigned species_mask);

/*
 * Pack positions and species for the AEV kernels: xyzs[i] = (x, y, z,
 * species index as int bits).  species_idx are positions in species_order.
 */
int fennol_pack_atoms(const float* coords, const int* species_idx, int natoms, float* xyzs,
                      void* stream);

/* AEV output encodings. */
#define FENNOL_AEV_F32 0     /* float32 rows */
#define FENNOL_AEV_BF16 1    /* bfloat16 rows */
#define FENNOL_AEV_BF16X2 2  /* bfloat16 hi rows + bfloat16 lo rows (x ~= hi + lo) */
#define FENNOL_AEV_F16X2 3   /* float16 hi rows + float16 lo rows (x ~= hi + lo, ~22 bits) */

/*
 * ANIAEV forward.  Replaces ANIAEV.__call__ (embeddings/ani.py:47-142) with
 * the graph processors it reads (GraphProcessor preprocessing.py:719-777,
 * GraphFilterProcessor :979-1043, GraphAngularExtension :1085-1276,
 * GraphAngleProcessor :1294-1317, SwitchFunction misc/misc.py:617-716).
 * nbr_* is the radial list (cutoff p->radial_cutoff); the angular neighbours
 * (d^2 < angular_cutoff^2 with the reference's float32 arithmetic) and all
 * their unordered pairs (the triplets) are formed on chip.
 * Row i of the output is written at row `atom_row[i]` of `out` (leading
 * dimension `ld` elements); columns [F, ld) are left untouched.
 */
int fennol_aev_forward(const float* xyzs, int natoms, const int* atom_sys, const float* sys_cell,
                       const int* nbr_j, const unsigned* nbr_shift, const int* nbr_count,
                       int capacity, const fennol_aev_params* p, const int* atom_row,
                       int out_kind, void* out, void* out_lo, int ld, int* status, void* stream);

/*
 * Adjoint of fennol_aev_forward: given dE/dAEV (float32 rows at atom_row,
 * leading dimension ld) accumulate forces -dE/dx into forces4[natoms*4]
 * (x, y, z, unused).  Replaces the reverse-mode transpose of the AEV
 * (jax.grad through ani.py and the graph processors, fennix.py:260-272).
 * forces4 must be zeroed (or hold other force terms) before the call.
 * daev must be 16-byte aligned and ld a multiple of 4 (FENNOL_ERR_INVALID
 * otherwise).
 */
int fennol_aev_backward(const float* xyzs, int natoms, const int* atom_sys,
                        const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                        const int* nbr_count, int capacity, const fennol_aev_params* p,
                        const int* atom_row, const float* daev, int ld, float* forces4,
                        int* status, void* stream);

/*
 * A forward/adjoint pair that shares the per-centre staging.  Both kernels
 * first gather each centre's row, compute its edge vectors, distances and
 * cutoffs, and sort the neighbours by species (ani.py:47-142 and the graph
 * processors it reads); with these two calls the forward saves that staged
 * neighbourhood to `stage` and the adjoint of the same step reads it back
 * instead of recomputing it.  fennol_aev_forward_staged is fennol_aev_forward
 * plus the save; fennol_aev_backward_staged is fennol_aev_backward (same
 * result) reading `stage`, which must come from fennol_aev_forward_staged on
 * the same positions, lists, capacity and parameters, with no other call
 * writing it in between.  `stage` is device memory of
 * fennol_aev_stage_bytes(natoms, capacity) bytes, 16-byte aligned.
 */
size_t fennol_aev_stage_bytes(int natoms, int capacity);
int fennol_aev_forward_staged(const float* xyzs, int natoms, const int* atom_sys,
                              const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                              const int* nbr_count, int capacity, const fennol_aev_params* p,
                              const int* atom_row, int out_kind, void* out, void* out_lo, int ld,
                              void* stage, size_t stage_bytes, int* status, void* stream);
int fennol_aev_backward_staged(const float* xyzs, int natoms, const int* atom_sys,
                               const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                               const int* nbr_count, int capacity, const fennol_aev_params* p,
                               const int* atom_row, const float* daev, int ld, float* forces4,
                               const void* stage, int* status, void* stream);

/*
 * fennol_aev_backward that also writes, per centre atom i, the 3x3 sum over
 * its edges of r_ij (x) dE/dr_ij (atom_virial, float32 [natoms*9], row-major
 * a,b = r_a * g_b).  Summed per system (fennol_virial_reduce) this is the
 * reference's virial_tensor = dE/dS of a homogeneous deformation
 * x -> x S, cell -> cell S at S = 1 (fennix.py:320-347).
 */
int fennol_aev_backward_virial(const float* xyzs, int natoms, const int* atom_sys,
                               const float* sys_cell, const int* nbr_j, const unsigned* nbr_shift,
                               const int* nbr_count, int capacity, const fennol_aev_params* p,
                               const int* atom_row, const float* daev, int ld, float* forces4,
                               float* atom_virial, int* status, void* stream);

/*
 * Forward-mode tangent of the AEV: out[atom_row[i]*ld + f] = sum_k
 * dAEV_i,f/dx_k . du_k for a displacement field du4 (float32 [natoms*4],
 * x, y, z, unused).  No counterpart call in the reference: jax.grad over a
 * loss that contains forces (training/utils.py:140-525) forms this product
 * inside XLA's second-order transpose; the training gradient uses it to
 * differentiate sum_i <dE/dAEV_i, t_i> with respect to the network
 * parameters.  float32 output, same row layout as fennol_aev_forward.
 */
int fennol_aev_tangent(const float* xyzs, int natoms, const int* atom_sys, const float* sys_cell,
                       const int* nbr_j, const unsigned* nbr_shift, const int* nbr_count,
                       int capacity, const fennol_aev_params* p, const int* atom_row,
                       const float* du4, float* out, int ld, int* status, void* stream);

/* ------------------------------------------------------------------------ */
/* Species-indexed MLP                                                       */
/* ------------------------------------------------------------------------ */

#define FENNOL_MLP_FP32 0     /* float32 CUDA-core GEMMs */
#define FENNOL_MLP_BF16 1     /* tcgen05 BF16 x BF16, FP32 accumulate */
#define FENNOL_MLP_BF16X2 2   /* activations split hi+lo BF16 (2 MMAs); weights as BF16 */
#define FENNOL_MLP_BF16X3 3   /* activations and weights split (3 MMAs) */
/* FP16 forms for float32 weights: activations and power-of-two-scaled weights
 * split into float16 hi + lo (about 22 bits each).  The forward GEMMs take
 * three products (A_hi W_hi + A_lo W_hi + A_hi W_lo); the input-gradient GEMMs
 * take one (G_hi W_hi, F16X3X1) or two (G_hi W_hi + G_hi W_lo, F16X3X2). */
#define FENNOL_MLP_F16X3X1 4
#define FENNOL_MLP_F16X3X2 5

#define FENNOL_MLP_LAYERS 4

/*
 * Packed weights of an ensemble of per-species networks
 * (FullyConnectedNet, misc/nets.py:13-102, inside SpeciesIndexNet :301-426).
 * A "group" is (model m, species s), index g = m*n_species + s.
 * dims[0..4] are the zero-padded widths (multiples of 64 except dims[4]=1):
 * 1024, 256, 192, 192, 1 for the ANI-2x network 1008-256-192-160-1.
 *   w32[l]: float32 [G][dims[l]][dims[l+1]]  (kernel, zero padded)
 *   b32[l]: float32 [G][dims[l+1]]
 *   wt_hi[l], wt_lo[l]: bfloat16 [G][dims[l+1]][dims[l]]  (kernel^T, K-major)
 *   w_hi[l], w_lo[l]:   bfloat16 [G][dims[l]][dims[l+1]]  (kernel, K-major for the
 *                        input-gradient GEMMs); used for l = 0..2.
 * bf16 pointers may be NULL for FENNOL_MLP_FP32; *_lo may be NULL unless
 * FENNOL_MLP_BF16X3.
 * For FENNOL_MLP_F16X3X1 / F16X3X2 the four split copies are float16 and hold
 * kernel * f16_scale[g*4 + l] (l = 0..2), a power of two chosen per group and
 * layer so that the largest entry lies in [1, 2); f16_scale[g*4 + 3] is the
 * power of two applied to the last layer's kernel inside the input-gradient
 * GEMMs.  wt_lo is required for both FP16 forms, w_lo for F16X3X2 only.
 * f16_scale (16-byte aligned) may be NULL for the other forms.
 */
typedef struct fennol_mlp_weights {
  int n_models;
  int n_species;
  int dims[5];
  float celu_alpha;
  const float* w32[FENNOL_MLP_LAYERS];
  const float* b32[FENNOL_MLP_LAYERS];
  const void* wt_hi[FENNOL_MLP_LAYERS];
  const void* wt_lo[FENNOL_MLP_LAYERS];
  const void* w_hi[FENNOL_MLP_LAYERS];
  const void* w_lo[FENNOL_MLP_LAYERS];
  const float* f16_scale;
} fennol_mlp_weights;

/* Workspace of fennol_mlp_energy_grad for `rows` padded rows, in bytes. */
size_t fennol_mlp_workspace_bytes(int precision, int rows, int n_models,
                                  const fennol_mlp_weights* w);

/*
 * Energies and input gradients of the species networks.  Replaces the
 * SpeciesIndexNet forward (nets.py:397-417), its jax.grad transpose and the
 * ensemble mean.  Rows are grouped by species in tiles of 128: tile t covers
 * rows [tile_row[t], tile_row[t]+128) of species tile_species[t] (padding
 * rows must hold zeros).  Inputs: x (AEV rows, ld = dims[0]; float32 for
 * FENNOL_MLP_FP32, float16 hi + lo for the FP16 forms, bfloat16 hi (+ lo)
 * otherwise).  The FP16 forms run only as the fused kernel (hidden widths
 * <= 256, input width a multiple of 256; FENNOL_ERR_UNSUPPORTED otherwise).  Outputs: e_rows[rows]
 * (ensemble-mean atomic energy) and dx[rows*dims[0]] (float32 dE/dAEV,
 * ensemble mean).
 */
int fennol_mlp_energy_grad(int precision, int rows, int ntiles, const int* tile_species,
                           const int* tile_row, const fennol_mlp_weights* w, const void* x,
                           const void* x_lo, float* e_rows, float* dx, void* workspace,
                           size_t workspace_bytes, void* stream);

/*
 * fennol_mlp_energy_grad for inputs whose columns are zero outside known
 * 64-column chunks.  No separate counterpart in the reference: SpeciesIndexNet
 * (nets.py:397-417) multiplies every column, and the ANIAEV columns of
 * species (pairs) absent from a batch are zero there too.  Bit c of
 * active_chunks says that columns [64c, 64c + 64) of x may be non-zero; the
 * caller guarantees that every other column is zero in every row (for AEV
 * rows, fennol_aev_active_chunks gives the mask of a species set).  The
 * fused tensor-core forms then skip the inactive K-chunks of the first layer
 * and write dx only in the active chunks (the other dx columns are left as
 * they were: the AEV adjoint reads only blocks of species present around
 * each centre); the other forms compute every column.  active_chunks == 0
 * is FENNOL_ERR_INVALID; ~0 is fennol_mlp_energy_grad.
 */
int fennol_mlp_energy_grad_active(int precision, int rows, int ntiles, const int* tile_species,
                                  const int* tile_row, const fennol_mlp_weights* w, const void* x,
                                  const void* x_lo, unsigned long long active_chunks, float* e_rows,
                                  float* dx, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Failure handling of the fused tensor-core MLP (no counterpart in the
 * reference).  Every wait inside the kernel on a shared-memory barrier gives
 * up after a time limit: the kernel then sets the int32 error word at the
 * start of its workspace to 1, ends all its roles, frees its tensor memory
 * and returns, so the context stays usable; the caller reads the word (and
 * clears it) after the launch.  Host only.
 *   fennol_mlp_wait_limit: the limit for later launches, in seconds
 *     (0 < seconds <= 60; default 2).
 *   fennol_mlp_inject_stall: the next `launches` fused launches start with a
 *     load producer that issues no copies, so the waits of the other roles
 *     run out (for tests of the timeout path; 0 clears).
 */
int fennol_mlp_wait_limit(double seconds);
int fennol_mlp_inject_stall(int launches);

/* ------------------------------------------------------------------------ */
/* Training-loss gradient                                                    */
/* ------------------------------------------------------------------------ */

/*
 * One species network per species, as the training gradient reads it
 * (unpadded FullyConnectedNet layers, misc/nets.py:13-102):
 *   w[l][s]: kernel [dims[l]][dims[l+1]] row-major, b[l][s]: bias [dims[l+1]];
 *   gw[l][s], gb[l][s]: outputs, same layouts.  dims = 1008, 256, 192, 160, 1
 *   for ANI-2x (dims[4] must be 1).  is_double selects float64 buffers and
 *   arithmetic, otherwise float32.  Pointers of species without rows may be NULL.
 */
typedef struct fennol_net_train {
  int n_species; /* <= 8 */
  int dims[5];
  float celu_alpha;
  int is_double;
  const void* w[FENNOL_MLP_LAYERS][8];
  const void* b[FENNOL_MLP_LAYERS][8];
  void* gw[FENNOL_MLP_LAYERS][8];
  void* gb[FENNOL_MLP_LAYERS][8];
} fennol_net_train;

/* Workspace of fennol_net_loss_grad for host_rows[s] rows per species, in bytes. */
size_t fennol_net_loss_grad_workspace_bytes(const fennol_net_train* net, const int* host_rows);

/*
 * Network part of the training-loss parameter gradient.  Replaces the
 * network half of jax.value_and_grad over a loss with forces
 * (training/utils.py:140-525, :508): for each species s, the gradient with
 * respect to its kernels and biases of
 *     sum over its rows r of  c_row[r] f_s(x_r) - <grad f_s(x_r), t_r>,
 * where x (AEV rows) and t (their tangents along dL/dF, fennol_aev_tangent)
 * are [rows][ld] in the species-sorted layout, species s owning rows
 * [host_row0[s], host_row0[s] + host_rows[s]), and c_row[r] = dL/dE of row r's
 * system.  CELU first and second derivatives are included.  All buffers in
 * the sweep's type (float32 or float64); workspace 256-byte aligned.  Each
 * stage is one grouped launch over the species; no host synchronisation.
 */
int fennol_net_loss_grad(const fennol_net_train* net, const int* host_row0, const int* host_rows,
                         const void* x, const void* t, int ld, const void* c_row, void* workspace,
                         size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Reductions and outputs                                                    */
/* ------------------------------------------------------------------------ */

/* Workspace of fennol_energy_reduce, in bytes.  It must be zero-filled
 * before its first use; every call leaves it ready for the next one. */
size_t fennol_energy_workspace_bytes(int natoms, int nsys);

/*
 * Per-system energies in float64: energy[b] = scale * sum_{i in b}
 * e_rows[atom_row[i]] (fixed summation order: 1024-atom chunks from the
 * system's first atom, then the chunk sums in order, so a system's energy
 * does not depend on the other systems of the batch).  One kernel launch.
 * Replaces the segment_sum of FENNIX.total_energy (fennix.py:218-258).
 * e_atom (float64 [natoms], may be NULL) receives scale * per-atom energies
 * in input order.  Calls that share a workspace must be stream-ordered.
 */
int fennol_energy_reduce(const float* e_rows, const int* atom_row, int natoms,
                         const int* sys_start, int nsys, double scale, double* energy,
                         double* e_atom, void* workspace, size_t workspace_bytes, void* stream);

/* forces[i*3+k] = scale * forces4[i*4+k] (float32 output). */
int fennol_forces_finalize(const float* forces4, int natoms, float scale, float* forces,
                           void* stream);

/* virial[b*9 + k] = scale * sum of atom_virial[i*9 + k] over the atoms of
 * system b (float64, fixed order). */
int fennol_virial_reduce(const float* atom_virial, int natoms, const int* sys_start, int nsys,
                         double scale, double* virial, void* stream);

/* ------------------------------------------------------------------------ */
/* Molecular dynamics                                                        */
/* ------------------------------------------------------------------------ */

/*
 * One BAOAB-style step of FeNNol's integrator (md/integrate.py:286-294) in
 * float64:  v += dt/m * F;  x += dt/2 v;  v = a1 v + a2_i xi (Langevin,
 * thermostats.py:56-120; NVE when a1 == 1 and a2 == NULL);  x += dt/2 v.
 * Units: A, ps, kcal/mol; inv_mass[i] = 1/m_i in the same system; forces4
 * holds -dE/dx in model units and is multiplied by force_scale.  xi are
 * standard normal numbers from a counter-based Philox4x32-10 stream keyed by
 * (seed, *step_counter, atom); step_counter is a device uint64 that the call
 * increments after the step, so a CUDA graph of the step draws new noise on
 * every replay (required when a2 != NULL).  Also writes float32 positions
 * (coords) and packed xyzs for the next force call, and sets
 * *rebuild_flag = 1 when an atom moved more than half the skin since the
 * last rebuild (x_ref).  If rebuild_flag is NULL no displacement check is done.
 */
int fennol_md_step(int natoms, double dt, double* x, double* v, const double* inv_mass,
                   const float* forces4, double force_scale, double a1, const double* a2,
                   unsigned long long seed, unsigned long long* step_counter, float* coords,
                   const int* species_idx, float* xyzs, const double* x_ref, double half_skin,
                   int* rebuild_flag, void* stream);

/*
 * fennol_md_step for a batch of independent systems (no counterpart in the
 * reference, whose MD driver integrates one system; used by the serving
 * loop).  Same update; the Langevin noise of atom i in system b = atom_sys[i]
 * comes from the Philox block keyed by sys_seed[b] at counter
 * (i - sys_start[b], sys_step[b]), so each system's trajectory is the same
 * whichever systems share the batch.  sys_step[0..nsys) (device uint64) is
 * incremented after the step.  Atoms [0, natoms) must belong to systems
 * [0, nsys).
 */
int fennol_md_step_systems(int natoms, int nsys, double dt, double* x, double* v,
                           const double* inv_mass, const float* forces4, double force_scale,
                           double a1, const double* a2, const int* atom_sys, const int* sys_start,
                           const unsigned long long* sys_seed, unsigned long long* sys_step,
                           float* coords, const int* species_idx, float* xyzs,
                           const double* x_ref, double half_skin, int* rebuild_flag, void* stream);

/* After a rebuild: x_ref = x and *rebuild_flag = 0 (both device). */
int fennol_md_mark_rebuilt(int natoms, const double* x, double* x_ref, int* rebuild_flag,
                           void* stream);

/*
 * Conditional neighbour-list update inside a CUDA graph of MD steps.  The
 * reference decides between a full rebuild and a skin update on the host
 * every step (md/integrate.py:515-565); these two calls let a captured step
 * make that decision on the device from the displacement flag that
 * fennol_md_step sets.  While `stream` is being captured,
 * fennol_capture_if_begin enqueues a one-thread kernel that copies
 * (*flag != 0) into the condition of an IF node added after it; the work the
 * caller then enqueues on `body_stream` (its own stream, not capturing) until
 * fennol_capture_if_end is captured into the body of that node, which a
 * replay runs only when the flag was set.  Work enqueued on `stream` after
 * fennol_capture_if_begin depends on the IF node.  Returns
 * FENNOL_ERR_UNSUPPORTED (enqueuing nothing) when `stream` is not capturing.
 */
int fennol_capture_if_begin(void* stream, const int* flag, void* body_stream);
int fennol_capture_if_end(void* body_stream);

/*
 * status[FENNOL_ST_NONFINITE] = 1 when any element of the nbuf (<= 4) device
 * buffers is a NaN or an infinity; buffer k holds host_counts[k] float32
 * (host_is_double[k] == 0) or float64 values.  One launch.  The host arrays
 * are read during the call.  Plays the part of the reference MD driver's NaN
 * check of positions and velocities (md/dynamic.py:204-208, 595-597), and
 * also checks energies and forces of single points.
 */
int fennol_check_finite(int nbuf, const void* const* host_ptrs, const size_t* host_counts,
                        const int* host_is_double, int* status, void* stream);

/* kinetic[0] = 0.5 * sum m v^2 (float64, deterministic order). */
int fennol_md_kinetic(int natoms, const double* v, const double* inv_mass, double* kinetic,
                      void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FENNOL_B200_H */
