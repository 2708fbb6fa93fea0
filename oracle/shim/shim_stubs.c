/* Test-infrastructure stubs that let the reference's driver.c,
 * orbital_integration.c and types_definition.c link into the oracle library
 * without MKL, cpy-dataio or the reference's text I/O (dataio.c).  Only
 * mctdhb_propagate_step (driver.c:159-201) is used from driver.c; the
 * recording and screen-monitor helpers of integration_driver
 * (driver.c:204-333) are outside the oracle and abort if reached. */
#include "assistant/dataio.h"
#include "cpydataio.h"
#include "mkl_dfti.h"
#include <stdio.h>
#include <stdlib.h>

static void
not_in_oracle(const char* name)
{
    fprintf(stderr, "oracle: %s is outside the compiled reference path\n", name);
    abort();
}

MKL_LONG DftiCreateDescriptor(DFTI_DESCRIPTOR_HANDLE* h, int p, int d, MKL_LONG n, ...)
{
    (void) p; (void) d; (void) n;
    *h = NULL;
    return 0;
}
MKL_LONG DftiSetValue(DFTI_DESCRIPTOR_HANDLE h, int param, ...)
{
    (void) h; (void) param;
    return 0;
}
MKL_LONG DftiCommitDescriptor(DFTI_DESCRIPTOR_HANDLE h) { (void) h; return 0; }
MKL_LONG DftiComputeForward(DFTI_DESCRIPTOR_HANDLE h, void* x, ...)
{
    (void) h; (void) x;
    not_in_oracle("DftiComputeForward");
    return 1;
}
MKL_LONG DftiComputeBackward(DFTI_DESCRIPTOR_HANDLE h, void* x, ...)
{
    (void) h; (void) x;
    not_in_oracle("DftiComputeBackward");
    return 1;
}
MKL_LONG DftiFreeDescriptor(DFTI_DESCRIPTOR_HANDLE* h) { (void) h; return 0; }
char* DftiErrorMessage(MKL_LONG s) { (void) s; return "dfti shim"; }

void
cmat_print(uint32_t m, uint32_t n, double complex** a)
{
    for (uint32_t i = 0; i < m; i++)
    {
        for (uint32_t j = 0; j < n; j++)
            printf(" (%+.6e%+.6ej)", creal(a[i][j]), cimag(a[i][j]));
        printf("\n");
    }
}
void rarr_column_txt(char f[], char fmt[], uint32_t n, double* v)
{
    (void) f; (void) fmt; (void) n; (void) v;
    not_in_oracle("rarr_column_txt");
}

void toggle_new_append_files() { not_in_oracle("toggle_new_append_files"); }
void set_output_fname(char p[], RecordDataType r, char* f)
{
    (void) p; (void) r; (void) f;
    not_in_oracle("set_output_fname");
}
void screen_integration_monitor_columns() { not_in_oracle("screen_integration_monitor_columns"); }
void screen_integration_monitor(MCTDHBDataStruct m)
{
    (void) m;
    not_in_oracle("screen_integration_monitor");
}
void append_processed_state(char p[], ManyBodyState s)
{
    (void) p; (void) s;
    not_in_oracle("append_processed_state");
}
void record_raw_state(char p[], ManyBodyState s)
{
    (void) p; (void) s;
    not_in_oracle("record_raw_state");
}
void record_time_interaction(char p[], OrbitalEquation e, uint16_t r)
{
    (void) p; (void) e; (void) r;
    not_in_oracle("record_time_interaction");
}
void append_timestep_potential(char p[], OrbitalEquation e)
{
    (void) p; (void) e;
    not_in_oracle("append_timestep_potential");
}
void record_time_array(char p[], double a, double b, uint16_t r)
{
    (void) p; (void) a; (void) b; (void) r;
    not_in_oracle("record_time_array");
}
