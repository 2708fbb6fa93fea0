/* Test-infrastructure shim for MKL DFTI.  The FFT paths of the reference
 * (calculus.c dxFFT/d2xFFT, split_linear_orbitals.c spectral propagator) are
 * outside the configurational hot path; the descriptor calls made at
 * workspace construction (types_definition.c get_orbital_workspace) succeed
 * as no-ops and any actual transform aborts loudly. */
#ifndef ORACLE_SHIM_MKL_DFTI_H
#define ORACLE_SHIM_MKL_DFTI_H
#include "mkl_types.h"

typedef void* DFTI_DESCRIPTOR_HANDLE;

enum DFTI_CONFIG_PARAM
{
    DFTI_FORWARD_SCALE = 4,
    DFTI_BACKWARD_SCALE = 5
};
enum DFTI_CONFIG_VALUE
{
    DFTI_COMPLEX = 32,
    DFTI_DOUBLE = 36
};

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, int prec, int dom,
                              MKL_LONG dim, ...);
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, int param, ...);
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h);
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void* x, ...);
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void* x, ...);
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h);
char*    DftiErrorMessage(MKL_LONG status);
#endif
