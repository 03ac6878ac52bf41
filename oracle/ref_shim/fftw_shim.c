/* Definitions behind the FFTW shim (see fftw3.h in this directory). */
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"

void *fftw_malloc(size_t n) {
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 1) != 0) return NULL;
    return p;
}

void fftw_free(void *p) { free(p); }

static void unavailable(const char *what) {
    fprintf(stderr, "oracle build: %s called, but PME is not part of the 2b/3b oracle\n", what);
    abort();
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags) {
    (void)n; (void)in; (void)out; (void)flags;
    unavailable("fftw_plan_dft_r2c_1d");
    return NULL;
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags) {
    (void)n; (void)in; (void)out; (void)flags;
    unavailable("fftw_plan_dft_c2r_1d");
    return NULL;
}
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)n; (void)in; (void)out; (void)sign; (void)flags;
    unavailable("fftw_plan_dft_1d");
    return NULL;
}
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
    (void)p; (void)in; (void)out;
    unavailable("fftw_execute_dft_r2c");
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
    (void)p; (void)in; (void)out;
    unavailable("fftw_execute_dft_c2r");
}
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
    (void)p; (void)in; (void)out;
    unavailable("fftw_execute_dft");
}
void fftw_destroy_plan(fftw_plan p) { (void)p; }
void fftw_cleanup(void) {}
