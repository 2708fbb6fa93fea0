// batch_m4.cu -- batched H.C and density kernels for 4 orbitals
#include "batch_tmpl.cuh"
namespace mctdhb {
template int hcp_batch_launch<4>(const BatchSlot*, const BatchTile*, const BatchTile*, const int*,
                                 int, int, int, cudaStream_t);
template int gram_batch_launch<4>(const BatchSlot*, const BatchTile*, const int*, const int*,
                                  const int*, int, cudaStream_t);
template int batch_prepare<4>();
}  // namespace mctdhb
