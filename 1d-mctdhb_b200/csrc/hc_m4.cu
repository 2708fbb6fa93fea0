// H.C kernel instantiation for 4 orbitals (own translation unit: parallel build)
#include "hc_tmpl.cuh"
#include "pairhc_tmpl.cuh"
namespace mctdhb {
template int hc_launch_tmpl<4>(const SpaceView&, const double2*, double2*, const double2*,
                                const HcEpilogue&, int, cudaStream_t);
template int hcp_apply_tmpl<4>(const SpaceView&, const double2*, double2*, const HcEpilogue&,
                                 int, int, cudaStream_t);
template int hcp_prepare_tmpl<4>();
}
