// density-matrix kernel instantiation for 5 orbitals (own translation unit)
#include "dens_tmpl.cuh"
namespace mctdhb {
template int dens_launch_tmpl<5>(const SpaceView&, const double2*, double2*, int, int,
                                  cudaStream_t);
}
