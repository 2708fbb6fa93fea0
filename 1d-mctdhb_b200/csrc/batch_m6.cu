// batch_m6.cu -- batched H.C and density kernels for 6 orbitals
#include "batch_tmpl.cuh"
namespace mctdhb {
template int hc_batch_launch<6>(const BatchSlot*, const BatchTile*, const int*, const int*, int,
                                cudaStream_t);
template int dens_batch_launch<6>(const BatchSlot*, const BatchTile*, const int*, const int*,
                                  cudaStream_t);
}  // namespace mctdhb
