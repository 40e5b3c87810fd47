/*
 * Project-written stand-in for the small subset of the FFTW3 API that the reference's CPU sources
 * call (DCT.cpp, FFT.cpp).  TEST INFRASTRUCTURE ONLY: it exists so those unmodified reference
 * sources can be compiled here (no FFTW in this image) and used as a checker under oracle/_ref.
 *
 * Semantics follow the FFTW3 manual: REDFT10 is the unnormalised DCT-II
 * (Y_k = 2 sum_j X_j cos(pi (2j+1) k / 2n)), REDFT01 the unnormalised DCT-III
 * (Y_k = X_0 + 2 sum_{j>0} X_j cos(pi j (2k+1) / 2n)), and the complex DFT is
 * Y_k = sum_j X_j exp(sign * 2 pi i jk / n), all applied separably over the dimensions of a
 * row-major array, in double precision.  The DCTs run in O(n log n) on the plan's thread count
 * (fftw_plan_with_nthreads); the complex DFTs are evaluated directly.  Planning flags and wisdom
 * are accepted and ignored (wisdom is never written to disk).
 */
#ifndef BINDER_ORACLE_FFTW_SHIM_H
#define BINDER_ORACLE_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct binder_shim_plan *fftw_plan;

typedef enum {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out, fftw_r2r_kind k0,
                           fftw_r2r_kind k1, unsigned flags);
fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double *in, double *out, fftw_r2r_kind k0,
                           fftw_r2r_kind k1, fftw_r2r_kind k2, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
int fftw_export_wisdom_to_filename(const char *filename);
int fftw_import_wisdom_from_filename(const char *filename);

#ifdef __cplusplus
}
#endif
#endif
