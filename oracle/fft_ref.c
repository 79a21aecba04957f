/* Reference FFT for the oracles (TEST INFRASTRUCTURE, never linked into the
 * product library).
 *
 * A plain mixed-radix Cooley-Tukey decimation-in-time transform written from
 * the DFT definition X[k] = sum_j x[j] exp(sign * 2 pi i j k / n), recursive
 * over the smallest prime factor, with a direct DFT for each factor.  No
 * normalisation in either direction (the convention FFTW documents and the
 * reference relies on at src/System/PBC.cpp:435-444 and :566-574).
 *
 * Not re-entrant (one cached twiddle table).
 * Used by the FFTW-API shim that lets the unmodified reference link here
 * (fftw_shim.c) and by the FP64 restatement (mdf_oracle.c).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fft_ref.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

static int smallest_factor(int n)
{
    if (n % 4 == 0) return 4;
    if (n % 2 == 0) return 2;
    for (int p = 3; p * p <= n; p += 2)
        if (n % p == 0) return p;
    return n;
}

/* out[k], k<n, from x[0], x[s], x[2s], ...; tw = exp(sign 2 pi i j / N0) table,
 * N0 = n * tstride. */
static void fft_rec(const double *x, double *out, int n, long s, int sign,
                    const double *tw, long tstride, double *scratch)
{
    if (n == 1) {
        out[0] = x[0];
        out[1] = x[1];
        return;
    }
    int p = smallest_factor(n);
    int m = n / p;
    for (int q = 0; q < p; ++q)
        fft_rec(x + 2 * (long)q * s, out + 2 * (long)q * m, m, s * p, sign, tw, tstride * p, scratch);
    /* combine: X[k + t m] = sum_r W_n^{r(k + t m)} Y_r[k] */
    double *y = scratch;            /* 2p doubles */
    double *z = scratch + 2 * p;    /* 2p doubles */
    long N0 = (long)n * tstride;
    for (int k = 0; k < m; ++k) {
        for (int r = 0; r < p; ++r) {
            long e = ((long)r * k % n) * tstride;
            double wr = tw[2 * e], wi = tw[2 * e + 1];
            double ar = out[2 * ((long)r * m + k)], ai = out[2 * ((long)r * m + k) + 1];
            y[2 * r] = ar * wr - ai * wi;
            y[2 * r + 1] = ar * wi + ai * wr;
        }
        for (int t = 0; t < p; ++t) {
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; ++r) {
                long e = ((long)r * t % p) * m * tstride;
                e %= N0;
                double wr = tw[2 * e], wi = tw[2 * e + 1];
                sr += y[2 * r] * wr - y[2 * r + 1] * wi;
                si += y[2 * r] * wi + y[2 * r + 1] * wr;
            }
            z[2 * t] = sr;
            z[2 * t + 1] = si;
        }
        for (int t = 0; t < p; ++t) {
            out[2 * ((long)t * m + k)] = z[2 * t];
            out[2 * ((long)t * m + k) + 1] = z[2 * t + 1];
        }
    }
}

/* per-(n, sign) twiddle table and work buffers, reused across lines */
static double *g_tw = 0, *g_in = 0, *g_out = 0, *g_scr = 0;
static int g_n = 0, g_sign = 0;

static void prepare(int n, int sign)
{
    if (n == g_n && sign == g_sign) return;
    free(g_tw); free(g_in); free(g_out); free(g_scr);
    g_tw = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    g_in = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    g_out = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    g_scr = (double *)malloc(sizeof(double) * 4 * (size_t)(n + 4));
    for (int j = 0; j < n; ++j) {
        double a = 2.0 * M_PI * (double)j / (double)n;
        g_tw[2 * j] = cos(a);
        g_tw[2 * j + 1] = sign * sin(a);
    }
    g_n = n;
    g_sign = sign;
}

void fft_ref_1d(double *data, int n, long stride, int sign)
{
    /* in-place complex transform of data[j*stride], j<n (interleaved re/im) */
    prepare(n, sign);
    for (int j = 0; j < n; ++j) {
        g_in[2 * j] = data[2 * (long)j * stride];
        g_in[2 * j + 1] = data[2 * (long)j * stride + 1];
    }
    fft_rec(g_in, g_out, n, 1, sign, g_tw, 1, g_scr);
    for (int j = 0; j < n; ++j) {
        data[2 * (long)j * stride] = g_out[2 * j];
        data[2 * (long)j * stride + 1] = g_out[2 * j + 1];
    }
}

void fft_ref_3d(double *c, int nx, int ny, int nz, int sign)
{
    /* complex [nx][ny][nz] in place */
    for (long i = 0; i < (long)nx * ny; ++i)
        fft_ref_1d(c + 2 * i * nz, nz, 1, sign);
    for (int i = 0; i < nx; ++i)
        for (int k = 0; k < nz; ++k)
            fft_ref_1d(c + 2 * ((long)i * ny * nz + k), ny, nz, sign);
    for (long jk = 0; jk < (long)ny * nz; ++jk)
        fft_ref_1d(c + 2 * jk, nx, (long)ny * nz, sign);
}

void fft_ref_r2c_3d(const double *in, double *out, int nx, int ny, int nz)
{
    long n = (long)nx * ny * nz;
    int nzc = nz / 2 + 1;
    double *c = (double *)calloc(2 * (size_t)n, sizeof(double));
    for (long i = 0; i < n; ++i) c[2 * i] = in[i];
    fft_ref_3d(c, nx, ny, nz, -1);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nzc; ++k) {
                long s = ((long)i * ny + j) * nz + k;
                long d = ((long)i * ny + j) * nzc + k;
                out[2 * d] = c[2 * s];
                out[2 * d + 1] = c[2 * s + 1];
            }
    free(c);
}

void fft_ref_c2r_3d(const double *in, double *out, int nx, int ny, int nz)
{
    long n = (long)nx * ny * nz;
    int nzc = nz / 2 + 1;
    double *c = (double *)calloc(2 * (size_t)n, sizeof(double));
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                long d = ((long)i * ny + j) * nz + k;
                if (k < nzc) {
                    long s = ((long)i * ny + j) * nzc + k;
                    c[2 * d] = in[2 * s];
                    c[2 * d + 1] = in[2 * s + 1];
                } else {
                    int ii = (nx - i) % nx, jj = (ny - j) % ny, kk = nz - k;
                    long s = ((long)ii * ny + jj) * nzc + kk;
                    c[2 * d] = in[2 * s];
                    c[2 * d + 1] = -in[2 * s + 1];
                }
            }
    fft_ref_3d(c, nx, ny, nz, +1);
    for (long i = 0; i < n; ++i) out[i] = c[2 * i];
    free(c);
}

void fft_ref_r2c_1d(const double *in, double *out, int n)
{
    double *c = (double *)calloc(2 * (size_t)n, sizeof(double));
    for (int i = 0; i < n; ++i) c[2 * i] = in[i];
    fft_ref_1d(c, n, 1, -1);
    for (int k = 0; k < n / 2 + 1; ++k) {
        out[2 * k] = c[2 * k];
        out[2 * k + 1] = c[2 * k + 1];
    }
    free(c);
}
