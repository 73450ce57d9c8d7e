// Library-level C entry points: version and the MLP dispatcher.
#include "mlp_common.cuh"

extern "C" const char* fennol_version(void) { return "fennol_b200 0.1 (sm_100a)"; }

static bool weights_ok(int precision, const fennol_mlp_weights* w) {
  if (!w || w->n_models < 1 || w->n_species < 1) return false;
  for (int l = 0; l < 4; ++l)
    if (w->dims[l] <= 0 || w->dims[l] % 64 != 0) return false;
  if (w->dims[4] != 1) return false;
  for (int l = 0; l < 4; ++l)
    if (!w->w32[l] || !w->b32[l]) return false;
  if (precision != FENNOL_MLP_FP32) {
    for (int l = 0; l < 3; ++l) {
      if (!w->wt_hi[l] || !w->w_hi[l]) return false;
      if (precision == FENNOL_MLP_BF16X3 && (!w->wt_lo[l] || !w->w_lo[l])) return false;
      if ((precision == FENNOL_MLP_F16X3X1 || precision == FENNOL_MLP_F16X3X2) && !w->wt_lo[l]) return false;
      if (precision == FENNOL_MLP_F16X3X2 && !w->w_lo[l]) return false;
    }
  }
  if ((precision == FENNOL_MLP_F16X3X1 || precision == FENNOL_MLP_F16X3X2) && !w->f16_scale) return false;
  return true;
}

extern "C" size_t fennol_mlp_workspace_bytes(int precision, int rows, int n_models,
                                             const fennol_mlp_weights* w) {
  if (rows < 0 || !w) return 0;
  if (precision == FENNOL_MLP_FP32) return fnl_mlp_simt_workspace(rows, w);
  return fnl_mlp_tc_workspace(precision, rows, n_models, w);
}

extern "C" int fennol_mlp_energy_grad_active(int precision, int rows, int ntiles, const int* tile_species,
                                             const int* tile_row, const fennol_mlp_weights* w, const void* x,
                                             const void* x_lo, unsigned long long active_chunks, float* e_rows,
                                             float* dx, void* workspace, size_t workspace_bytes, void* stream) {
  if (precision < FENNOL_MLP_FP32 || precision > FENNOL_MLP_F16X3X2) return FENNOL_ERR_INVALID;
  if (!weights_ok(precision, w)) return FENNOL_ERR_INVALID;
  if (rows < 0 || ntiles < 0 || rows % 128 != 0 || ntiles * 128 > rows) return FENNOL_ERR_INVALID;
  if (ntiles == 0) return FENNOL_OK;
  if (!tile_species || !tile_row || !x || !e_rows || !dx || !workspace) return FENNOL_ERR_INVALID;
  if (workspace_bytes < fennol_mlp_workspace_bytes(precision, rows, w->n_models, w))
    return FENNOL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == FENNOL_MLP_FP32)
    return fnl_mlp_simt(rows, ntiles, tile_species, tile_row, w, (const float*)x, e_rows, dx, workspace, st);
  if (precision != FENNOL_MLP_BF16 && !x_lo) return FENNOL_ERR_INVALID;
  if (!active_chunks) return FENNOL_ERR_INVALID;
  return fnl_mlp_tc(precision, rows, ntiles, tile_species, tile_row, w, x, x_lo, active_chunks, e_rows, dx,
                    workspace, workspace_bytes, st);
}

extern "C" int fennol_mlp_energy_grad(int precision, int rows, int ntiles, const int* tile_species,
                                      const int* tile_row, const fennol_mlp_weights* w, const void* x,
                                      const void* x_lo, float* e_rows, float* dx, void* workspace,
                                      size_t workspace_bytes, void* stream) {
  return fennol_mlp_energy_grad_active(precision, rows, ntiles, tile_species, tile_row, w, x, x_lo, ~0ull, e_rows,
                                       dx, workspace, workspace_bytes, stream);
}
