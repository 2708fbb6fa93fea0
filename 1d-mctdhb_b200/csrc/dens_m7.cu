// density-matrix kernel instantiation for 7 orbitals (own translation unit)
#include "dens_tmpl.cuh"
#include "gram_tmpl.cuh"
namespace mctdhb {
template int dens_launch_tmpl<7>(const SpaceView&, const double2*, double2*, int, int,
                                  cudaStream_t);
template int gram_apply_tmpl<7>(const SpaceView&, uint32_t, uint32_t, const double2*, double2*,
                                  double2*, double2*, cudaStream_t);
template int gram_prepare_tmpl<7>();
}
