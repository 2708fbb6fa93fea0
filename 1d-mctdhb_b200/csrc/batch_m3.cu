// batch_m3.cu -- batched H.C and density kernels for 3 orbitals
#include "batch_tmpl.cuh"
namespace mctdhb {
template int hcp_batch_launch<3>(const BatchSlot*, const BatchTile*, const BatchTile*, const int*,
                                 int, int, int, cudaStream_t);
template int gram_batch_launch<3>(const BatchSlot*, const BatchTile*, const int*, const int*,
                                  const int*, int, cudaStream_t);
template int batch_prepare<3>();
}  // namespace mctdhb
