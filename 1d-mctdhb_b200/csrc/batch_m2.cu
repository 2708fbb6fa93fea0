// batch_m2.cu -- batched H.C and density kernels for 2 orbitals
#include "batch_tmpl.cuh"
namespace mctdhb {
template int hcp_batch_launch<2>(const BatchSlot*, const BatchTile*, const BatchTile*, const int*,
                                 int, int, int, cudaStream_t);
template int gram_batch_launch<2>(const BatchSlot*, const BatchTile*, const int*, const int*,
                                  const int*, int, cudaStream_t);
template int batch_prepare<2>();
}  // namespace mctdhb
