// batch_m5.cu -- batched H.C and density kernels for 5 orbitals
#include "batch_tmpl.cuh"
namespace mctdhb {
template int hcp_batch_launch<5>(const BatchSlot*, const BatchTile*, const BatchTile*, const int*,
                                 int, int, int, cudaStream_t);
template int gram_batch_launch<5>(const BatchSlot*, const BatchTile*, const int*, const int*,
                                  const int*, int, cudaStream_t);
template int batch_prepare<5>();
}  // namespace mctdhb
