/* Build shim for compiling the reference library without FFTW.
 *
 * The reference's PME code (potential/electrostatics/helpme.h) includes
 * <fftw3.h> unconditionally, and its no-FFTW fallback does not compile
 * (helpme.h:1325 calls CleanupFFTW() without the argument its fallback
 * signature takes), so the oracle build defines HAVE_FFTWD=1 and supplies the
 * double-precision FFTW names helpme.h binds (helpme.h:1233-1243) plus the
 * allocation pair and flags.  The 2-body/3-body path never reaches PME; the
 * planner and executor entry points abort if anything ever calls them, and
 * the clean-up calls made by destructors are no-ops.  This is test
 * infrastructure, not part of the product.
 */
#ifndef MBX_ORACLE_FFTW3_SHIM_H
#define MBX_ORACLE_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct mbx_oracle_fftw_plan_s *fftw_plan;
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);
#ifdef __cplusplus
}
#endif
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#endif
