/* Minimal FFTW3-compatible declarations (TEST INFRASTRUCTURE).
 *
 * The reference includes FFTW3 3.3.10 from an absolute macOS path
 * (include/System/System.h:13, src/System/PBC.cpp:6) and calls exactly these
 * entry points (src/System/PBC.cpp:409-428, :443, :468-488, :573).  FFTW is
 * not installed here, so the oracle build links the reference against
 * fftw_shim.c instead.  Names and signatures follow FFTW's public API so the
 * reference sources compile unchanged; the implementation behind them is this
 * project's own (fft_ref.c).
 */
#ifndef MDF_FFTW3_SHIM_H
#define MDF_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef double fftw_complex[2];
typedef struct mdf_fftw_plan_s *fftw_plan;
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
#ifdef __cplusplus
}
#endif
#endif
