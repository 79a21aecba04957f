/* FFTW-API shim over fft_ref.c (TEST INFRASTRUCTURE: links the unmodified
 * reference here; see fftw3.h for why).  Plans only record their arguments;
 * execution is the unnormalised r2c / c2r transform with FFTW's half-complex
 * layout [n0][n1][n2/2+1]. */
#include <stdlib.h>
#include "fftw3.h"
#include "../fft_ref.h"

struct mdf_fftw_plan_s {
    int kind;       /* 0 r2c 3d, 1 c2r 3d, 2 r2c 1d */
    int n0, n1, n2;
    void *in, *out;
};

static fftw_plan mk(int kind, int n0, int n1, int n2, void *in, void *out)
{
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->kind = kind; p->n0 = n0; p->n1 = n1; p->n2 = n2; p->in = in; p->out = out;
    return p;
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags)
{
    (void)flags;
    return mk(0, n0, n1, n2, in, out);
}

fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags)
{
    (void)flags;
    return mk(1, n0, n1, n2, in, out);
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned flags)
{
    (void)flags;
    return mk(2, n, 1, 1, in, out);
}

void fftw_execute(const fftw_plan p)
{
    if (p->kind == 0)
        fft_ref_r2c_3d((const double *)p->in, (double *)p->out, p->n0, p->n1, p->n2);
    else if (p->kind == 1)
        fft_ref_c2r_3d((const double *)p->in, (double *)p->out, p->n0, p->n1, p->n2);
    else
        fft_ref_r2c_1d((const double *)p->in, (double *)p->out, p->n0);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
void *fftw_malloc(size_t n) { return malloc(n); }
void fftw_free(void *p) { free(p); }
