/* Reference FFT for the oracles (test infrastructure only). */
#ifndef MDF_ORACLE_FFT_REF_H
#define MDF_ORACLE_FFT_REF_H
#ifdef __cplusplus
extern "C" {
#endif
void fft_ref_1d(double *data, int n, long stride, int sign);
void fft_ref_3d(double *c, int nx, int ny, int nz, int sign);
void fft_ref_r2c_3d(const double *in, double *out, int nx, int ny, int nz);
void fft_ref_c2r_3d(const double *in, double *out, int nx, int ny, int nz);
void fft_ref_r2c_1d(const double *in, double *out, int n);
#ifdef __cplusplus
}
#endif
#endif
