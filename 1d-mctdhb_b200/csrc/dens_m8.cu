// density-matrix kernel instantiation for 8 orbitals (own translation unit)
#include "dens_tmpl.cuh"
namespace mctdhb {
template int dens_launch_tmpl<8>(const SpaceView&, const double2*, double2*, int, int,
                                  cudaStream_t);
}
