// mlp.cu -- learned far-field correction (filled in by the far-field work).
#include "internal.cuh"

void mlp_free(gvizCudaForce *h) {
  if (h->d_mlp) cudaFree(h->d_mlp);
  h->d_mlp = nullptr;
}
