/* Test-infrastructure shim for cpy-dataio (github.com/andriati-alex/cpy-dataio,
 * not vendored with the reference).  Only the two names reached by the files
 * the oracle compiles (orbital_integration.c:51, driver.c:320) are declared;
 * their bodies live in shim_stubs.c. */
#ifndef ORACLE_SHIM_CPYDATAIO_H
#define ORACLE_SHIM_CPYDATAIO_H
#include <complex.h>
#include <stdint.h>
void cmat_print(uint32_t m, uint32_t n, double complex** a);
void rarr_column_txt(char fname[], char fmt[], uint32_t n, double* v);
#endif
