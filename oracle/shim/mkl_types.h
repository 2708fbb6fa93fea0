/* Test-infrastructure shim: the two MKL scalar types the reference's
 * public header (include/mctdhb_types.h:17-18,44) names.  Layout-compatible
 * with MKL LP64 on Linux; only used to compile the reference oracle. */
#ifndef ORACLE_SHIM_MKL_TYPES_H
#define ORACLE_SHIM_MKL_TYPES_H
typedef struct
{
    double real, imag;
} MKL_Complex16;
typedef long MKL_LONG;
#endif
