// batch_m5.cu -- batched H.C and density kernels for 5 orbitals
#include "batch_tmpl.cuh"
namespace mctdhb {
template int hc_batch_launch<5>(const BatchSlot*, const BatchTile*, const int*, const int*, int,
                                cudaStream_t);
template int dens_batch_launch<5>(const BatchSlot*, const BatchTile*, const int*, const int*,
                                  cudaStream_t);
}  // namespace mctdhb
