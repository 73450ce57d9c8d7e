// Tensor-core (tcgen05) species MLP -- placeholder until the kernel lands.
#include "mlp_common.cuh"

size_t fnl_mlp_tc_workspace(int, int, int, const fennol_mlp_weights*) { return 0; }

int fnl_mlp_tc(int, int, int, const int*, const int*, const fennol_mlp_weights*, const void*, const void*,
               float*, float*, void*, size_t, cudaStream_t) {
  return FENNOL_ERR_UNSUPPORTED;
}
