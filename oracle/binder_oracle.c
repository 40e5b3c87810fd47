/*
 * FP64 CPU oracle for the BINDER hot path -- TEST INFRASTRUCTURE ONLY (see binder_oracle.h).
 *
 * Every function restates one piece of the reference CPU backend (ste93ste/BINDER) and cites the
 * file:line it follows.  Compiled with -ffp-contract=off so that expression-by-expression FP64
 * evaluation order (and therefore the Jacobian determinants) matches the reference bit for bit.
 */
#include "binder_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_D 3.14159265358979323846

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------------------------ */
/* Philox4x32-10, as published by Salmon et al. (SC'11): 10 rounds of the 4x32 bijection with  */
/* the multipliers M0 = 0xD2511F53, M1 = 0xCD9E8D57 and the Weyl key increments 0x9E3779B9,    */
/* 0xBB67AE85.  The CUDA path uses the identical function so draws agree exactly.             */
/* ------------------------------------------------------------------------------------------ */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint64_t p0 = (uint64_t)0xD2511F53u * (uint64_t)c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * (uint64_t)c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline void philox_draw(uint64_t seed, uint32_t index, uint32_t sweep, uint32_t tag,
                               uint32_t chain, uint32_t out[4]) {
    const uint32_t ctr[4] = {index, sweep, tag, chain};
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    orc_philox4x32_10(ctr, key, out);
}

/* uniform in (0,1) with 23 random bits: exactly representable in float and double */
static inline double u01_f24(uint32_t x) { return ((double)(x >> 9) + 0.5) * (1.0 / 8388608.0); }
/* uniform in (0,1) with 32 random bits (double) */
static inline double u01_d32(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

/* ------------------------------------------------------------------------------------------ */
/* cubic B-spline weights for offsets -1, 0, 1, 2 at fraction d in [0,1)                       */
/* BINDER/src/cpu/Spline.cpp:44-73                                                             */
/* ------------------------------------------------------------------------------------------ */
void orc_spline3(double d, double w[4]) {
    const double d2 = d * d, d3 = d2 * d;
    const double e = 1.0 - d, e2 = e * e, e3 = e2 * e;
    w[0] = e3 / 6.0;
    w[1] = 2.0 / 3.0 - d2 + d3 * 0.5;
    w[2] = 2.0 / 3.0 - e2 + e3 * 0.5;
    w[3] = d3 / 6.0;
}

/* Spline.cpp:9-41 (offsets, index offset) and :93-123 (orders 2 and 1), placed on the cubic
 * stencil of node offsets -1, 0, 1, 2: order 2 uses -1, 0, 1 around floor(p + 0.5), order 1 uses
 * 0, 1 around floor(p); the unused taps carry weight 0. */
static int g_spline_order = 3;
void orc_set_spline_order(int order) { g_spline_order = (order == 1 || order == 2) ? order : 3; }
int orc_get_spline_order(void) { return g_spline_order; }

/* Spline::spline(d) as the reference returns it: the weights of its own offsets (order 3:
 * -1..2, order 2: -1..1, order 1: 0..1), zero-filled to four */
void orc_spline(int order, double d, double w[4]) {
    if (order == 2) {
        const double a = -2.0 * d + 1.0, b = -2.0 * d - 1.0;
        w[0] = 0.125 * (a * a);
        w[1] = 0.75 - d * d;
        w[2] = 0.125 * (b * b);
        w[3] = 0.0;
    } else if (order == 1) {
        w[0] = 1.0 - d;
        w[1] = d;
        w[2] = 0.0;
        w[3] = 0.0;
    } else {
        orc_spline3(d, w);
    }
}

/* base node index of position p, and its four weights on the offsets -1 .. 2 */
static int spline_setup(double p, double w[4]) {
    const double f = floor(p + (g_spline_order == 2 ? 0.5 : 0.0)), d = p - f;
    double r[4];
    orc_spline(g_spline_order, d, r);
    if (g_spline_order == 1) {  /* offsets 0, 1 sit at stencil taps 1, 2 */
        w[0] = 0.0; w[1] = r[0]; w[2] = r[1]; w[3] = 0.0;
    } else {
        for (int t = 0; t < 4; ++t) w[t] = r[t];
    }
    return (int)f;
}

/* moving-image bin at a node; outside the moving grid the likelihood uses row 0
 * (BINDER/src/cpu/MILikelihood.cpp:46-48, :92-93) */
static inline int node_bin(const int *v, int x, int y, int z, int nxn, int nyn, int nzn) {
    if (x < 0 || y < 0 || z < 0 || x >= nxn || y >= nyn || z >= nzn) return 0;
    return v[((long)x * nyn + y) * nzn + z];
}

typedef struct {
    double w[64];
    int kbin[64];
    int node[64][3];
    int n;
    double S;
    int base[3];  /* the spline's base node index per axis */
} neigh_t;

/* weights B(y_j - d_i) * theta[v_j, u_i] for the 4x4x4 (3D) or 4x4 (2D) neighbourhood,
 * Registration.cpp:219-272 */
static void neighbourhood(const double *di, int ui, const int *v, const double *theta, int is2D,
                          int nxn, int nyn, int nzn, int L, neigh_t *nb) {
    double bx[4], by[4], bz[4] = {1.0, 1.0, 1.0, 1.0};
    const int ix = spline_setup(di[0], bx), iy = spline_setup(di[1], by);
    const int iz = is2D ? 0 : spline_setup(di[2], bz);
    nb->base[0] = ix; nb->base[1] = iy; nb->base[2] = iz;
    const int ZZ = is2D ? 1 : 4;
    int j = 0;
    double S = 0.0;
    for (int a = 0; a < 4; ++a) {
        const int X = ix + a - 1;
        for (int b = 0; b < 4; ++b) {
            const int Y = iy + b - 1;
            const double bxy = bx[a] * by[b];
            for (int c = 0; c < ZZ; ++c) {
                const int Z = is2D ? 0 : iz + c - 1;
                const int k = node_bin(v, X, Y, Z, nxn, nyn, nzn);
                const double w = bxy * bz[c] * theta[(long)k * L + ui];
                nb->w[j] = w;
                nb->kbin[j] = k;
                nb->node[j][0] = X; nb->node[j][1] = Y; nb->node[j][2] = Z;
                S += w;
                ++j;
            }
        }
    }
    nb->n = j;
    nb->S = S;
}

/* Registration.cpp:122-165 (E-step loop) and :219-330 (per voxel, sample == false) */
double orc_estep(const double *d, const int *u, const int *v, const double *theta,
                 int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
                 double *dream, double *hist, long long *degenerate) {
    const int is2D = (nz == 1);
    const int N = is2D ? 2 : 3;
    const long V = (long)nx * ny * nz;
    const int T = orc_get_threads();
    double *hist_t = (double *)calloc((size_t)T * K * L, sizeof(double));
    double mll = 0.0;
    long long deg = 0;
#pragma omp parallel num_threads(T) reduction(+ : mll, deg)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        double *h = hist_t + (size_t)tid * K * L;
        neigh_t nb;
#pragma omp for schedule(static)
        for (long i = 0; i < V; ++i) {
            const double *di = d + i * N;
            neighbourhood(di, u[i], v, theta, is2D, nxn, nyn, nzn, L, &nb);
            double *dr = dream + i * N;
            if (!(nb.S > 0.0)) {
                for (int n = 0; n < N; ++n) dr[n] = (double)nb.base[n];
                deg += 1;
                continue;
            }
            mll += -log(nb.S);
            double acc[3] = {0.0, 0.0, 0.0};
            for (int j = 0; j < nb.n; ++j) {
                const double p = nb.w[j] / nb.S;
                h[(long)nb.kbin[j] * L + u[i]] += p;
                for (int n = 0; n < N; ++n) acc[n] += p * (double)nb.node[j][n];
            }
            for (int n = 0; n < N; ++n) dr[n] = acc[n];
        }
    }
    memset(hist, 0, sizeof(double) * K * L);
    for (int t = 0; t < T; ++t)
        for (long q = 0; q < (long)K * L; ++q) hist[q] += hist_t[(size_t)t * K * L + q];
    free(hist_t);
    if (degenerate) *degenerate = deg;
    return mll;
}

/* MILikelihoodFilter::compute_likelihood (BINDER/src/cpu/MILikelihoodFilter.cpp:53-68): the
 * product over the M channels of theta[m][k_m][l_m], channel m of voxel i being u[i + m] and of
 * node j v[j + m] (the reference's indexing: the channel windows overlap), a node outside the
 * grid having bin 0 in every channel. */
double orc_mi_filter_likelihood(const double *theta, const int *u, const int *v, int K, int L,
                                int M, int nxn, int nyn, int nzn, long voxel, int x, int y, int z) {
    const long KL = (long)K * L;
    const int outside = x < 0 || y < 0 || z < 0 || x >= nxn || y >= nyn || z >= nzn;
    const long node = outside ? 0 : ((long)x * nyn + y) * nzn + z;
    double t = 1.0;
    for (int m = 0; m < M; ++m) {
        const int k = outside ? 0 : v[node + m];
        t *= theta[m * KL + (long)k * L + u[voxel + m]];
    }
    return t;
}

/* The EM E-step (Registration.cpp:219-330, sample == false) with the MI filter likelihood:
 * weights B(y_j - d_i) * prod_m theta[m][k_m(j)][u_m(i)], posterior mass added to every
 * channel's histogram (MILikelihoodFilter.cpp:110-124).  hist [M][K][L]. */
double orc_estep_filter(const double *d, const int *u, const int *v, const double *theta,
                        int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L, int M,
                        double *dream, double *hist, long long *degenerate) {
    const int is2D = (nz == 1);
    const int N = is2D ? 2 : 3;
    const long V = (long)nx * ny * nz;
    const long KL = (long)K * L;
    const int T = orc_get_threads();
    double *hist_t = (double *)calloc((size_t)T * M * KL, sizeof(double));
    double mll = 0.0;
    long long deg = 0;
#pragma omp parallel num_threads(T) reduction(+ : mll, deg)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        double *h = hist_t + (size_t)tid * M * KL;
#pragma omp for schedule(static)
        for (long i = 0; i < V; ++i) {
            const double *di = d + i * N;
            double bx[4], by[4], bz[4] = {1.0, 1.0, 1.0, 1.0};
            const int ix = spline_setup(di[0], bx), iy = spline_setup(di[1], by);
            const int iz = is2D ? 0 : spline_setup(di[2], bz);
            const int ZZ = is2D ? 1 : 4;
            double w[64];
            int nodes[64][3];
            int n = 0;
            double S = 0.0;
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b)
                    for (int c = 0; c < ZZ; ++c) {
                        const int X = ix + a - 1, Y = iy + b - 1, Z = is2D ? 0 : iz + c - 1;
                        w[n] = bx[a] * by[b] * bz[c] *
                               orc_mi_filter_likelihood(theta, u, v, K, L, M, nxn, nyn, nzn, i,
                                                        X, Y, Z);
                        nodes[n][0] = X; nodes[n][1] = Y; nodes[n][2] = Z;
                        S += w[n];
                        ++n;
                    }
            double *dr = dream + i * N;
            if (!(S > 0.0)) {
                dr[0] = ix; dr[1] = iy;
                if (!is2D) dr[2] = iz;
                deg += 1;
                continue;
            }
            mll += -log(S);
            double acc[3] = {0.0, 0.0, 0.0};
            for (int j = 0; j < n; ++j) {
                const double p = w[j] / S;
                const int X = nodes[j][0], Y = nodes[j][1], Z = nodes[j][2];
                const int outside = X < 0 || Y < 0 || Z < 0 || X >= nxn || Y >= nyn || Z >= nzn;
                const long node = outside ? 0 : ((long)X * nyn + Y) * nzn + Z;
                for (int m = 0; m < M; ++m) {
                    const int k = outside ? 0 : v[node + m];
                    h[m * KL + (long)k * L + u[i + m]] += p;
                }
                for (int q = 0; q < N; ++q) acc[q] += p * (double)nodes[j][q];
            }
            for (int q = 0; q < N; ++q) dr[q] = acc[q];
        }
    }
    memset(hist, 0, sizeof(double) * M * KL);
    for (int t = 0; t < T; ++t)
        for (long q = 0; q < M * KL; ++q) hist[q] += hist_t[(size_t)t * M * KL + q];
    free(hist_t);
    if (degenerate) *degenerate = deg;
    return mll;
}

/* Registration.cpp:278-307 (sample == true): categorical draw over the neighbourhood.
 * The draw is t = u * S and the first neighbour whose running sum reaches t is taken, which is
 * the reference's normalised-CDF test (random_number <= cumulative_probability). */
double orc_estep_sample(const double *d, const int *u, const int *v, const double *theta,
                        int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
                        uint64_t seed, uint32_t sweep, uint32_t chain,
                        double *dream, double *hist) {
    const int is2D = (nz == 1);
    const int N = is2D ? 2 : 3;
    const long V = (long)nx * ny * nz;
    const int T = orc_get_threads();
    double *hist_t = (double *)calloc((size_t)T * K * L, sizeof(double));
    double mll = 0.0;
#pragma omp parallel num_threads(T) reduction(+ : mll)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        double *h = hist_t + (size_t)tid * K * L;
        neigh_t nb;
#pragma omp for schedule(static)
        for (long i = 0; i < V; ++i) {
            const double *di = d + i * N;
            neighbourhood(di, u[i], v, theta, is2D, nxn, nyn, nzn, L, &nb);
            double *dr = dream + i * N;
            if (!(nb.S > 0.0)) {
                for (int n = 0; n < N; ++n) dr[n] = (double)nb.base[n];
                continue;
            }
            mll += -log(nb.S);
            uint32_t r[4];
            philox_draw(seed, (uint32_t)i, sweep, 1u, chain, r);
            const double t = u01_f24(r[0]) * nb.S;
            double cdf = 0.0;
            int pick = nb.n - 1;
            for (int j = 0; j < nb.n; ++j) {
                cdf += nb.w[j];
                if (cdf >= t) { pick = j; break; }
            }
            h[(long)nb.kbin[pick] * L + u[i]] += 1.0;
            for (int n = 0; n < N; ++n) dr[n] = (double)nb.node[pick][n];
        }
    }
    memset(hist, 0, sizeof(double) * K * L);
    for (int t = 0; t < T; ++t)
        for (long q = 0; q < (long)K * L; ++q) hist[q] += hist_t[(size_t)t * K * L + q];
    free(hist_t);
    return mll;
}

/* MILikelihood.cpp:71-86: theta <- (hist + alpha - 1) / row sum */
void orc_theta_map(double *th, int K, int L, double alpha) {
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        for (int l = 0; l < L; ++l) s += th[k * L + l] + alpha - 1.0;
        for (int l = 0; l < L; ++l) th[k * L + l] = (th[k * L + l] + alpha - 1.0) / s;
    }
}

/* MILikelihood.cpp:33-39 and :183-206: sum_k -log Dir(theta_k; alpha) */
double orc_dirichlet_cost(const double *th, int K, int L, double alpha) {
    double cost = 0.0;
    for (int k = 0; k < K; ++k) {
        double sum_alpha = 0.0;
        for (int l = 0; l < L; ++l) sum_alpha += alpha;
        double lp = lgamma(sum_alpha);
        for (int l = 0; l < L; ++l) lp -= lgamma(alpha);
        for (int l = 0; l < L; ++l) lp += (alpha - 1.0) * log(th[k * L + l]);
        cost += -lp;
    }
    return cost;
}

/* Gamma(shape, 1) by Marsaglia & Tsang (ACM TOMS 26(3), 2000), with the shape < 1 boost
 * Gamma(a) = Gamma(a+1) * U^(1/a).  Attempt j draws Philox ctr = {index, sweep, tag | j<<8, chain}:
 * words 0,1 -> Box-Muller normal, word 2 -> acceptance uniform, word 3 -> boost uniform.
 * Capped at 64 attempts (acceptance probability per attempt is > 0.95). */
double orc_gamma_sample(double shape, uint64_t seed, uint32_t index, uint32_t sweep,
                        uint32_t tag, uint32_t chain, int *capped) {
    const int small = shape < 1.0;
    const double a = small ? shape + 1.0 : shape;
    const double dd = a - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * dd);
    for (uint32_t att = 0; att < 64; ++att) {
        uint32_t r[4];
        philox_draw(seed, index, sweep, tag | (att << 8), chain, r);
        const double u1 = u01_d32(r[0]), u2 = u01_d32(r[1]);
        const double z = sqrt(-2.0 * log(u1)) * cos(2.0 * PI_D * u2);
        double vv = 1.0 + c * z;
        if (vv <= 0.0) continue;
        vv = vv * vv * vv;
        const double uu = u01_d32(r[2]);
        if (uu < 1.0 - 0.0331 * (z * z) * (z * z) ||
            log(uu) < 0.5 * z * z + dd * (1.0 - vv + log(vv))) {
            double g = dd * vv;
            if (small) g *= pow(u01_d32(r[3]), 1.0 / shape);
            return g;
        }
    }
    if (capped) *capped = 1;
    return dd;
}

/* MILikelihood.cpp:132-169: theta_k ~ Dirichlet(hist_k + alpha) */
int orc_dirichlet_sample(double *th, int K, int L, double alpha, uint64_t seed, uint32_t sweep,
                         uint32_t chain) {
    int capped_rows = 0;
    for (int k = 0; k < K; ++k) {
        double s = 0.0;
        int capped = 0;
        for (int l = 0; l < L; ++l) {
            const double g = orc_gamma_sample(th[k * L + l] + alpha, seed, (uint32_t)(k * L + l),
                                              sweep, 4u, chain, &capped);
            th[k * L + l] = g;
            s += g;
        }
        for (int l = 0; l < L; ++l) th[k * L + l] /= s;
        capped_rows += capped;
    }
    return capped_rows;
}

/* ------------------------------------------------------------------------------------------ */
/* orthonormal DCT-II (forward) / DCT-III (inverse) along each axis, as the FFTW REDFT10/01   */
/* plans with the scaling of BINDER/src/cpu/DCT.cpp:83-175                                     */
/* ------------------------------------------------------------------------------------------ */
static double *dct_matrix(int n) {
    double *C = (double *)malloc(sizeof(double) * n * n);
    for (int k = 0; k < n; ++k) {
        const double s = (k == 0) ? sqrt(1.0 / n) : sqrt(2.0 / n);
        for (int j = 0; j < n; ++j) {
            const long m = ((long)(2 * j + 1) * k) % (4L * n);
            C[k * n + j] = s * cos(PI_D * (double)m / (2.0 * n));
        }
    }
    return C;
}

/* y[.., k, ..] = sum_j M[k][j] x[.., j, ..] along an axis of length n with stride s */
static void apply_axis(const double *M, int n, int transpose, double *data, long outer, long s) {
    const int T = orc_get_threads();
#pragma omp parallel num_threads(T)
    {
        double *in = (double *)malloc(sizeof(double) * n);
#pragma omp for schedule(static)
        for (long o = 0; o < outer * s; ++o) {
            const long b = (o / s) * (long)n * s + (o % s);
            for (int j = 0; j < n; ++j) in[j] = data[b + (long)j * s];
            for (int k = 0; k < n; ++k) {
                double acc = 0.0;
                if (!transpose)
                    for (int j = 0; j < n; ++j) acc += M[k * n + j] * in[j];
                else
                    for (int j = 0; j < n; ++j) acc += M[j * n + k] * in[j];
                data[b + (long)k * s] = acc;
            }
        }
        free(in);
    }
}

void orc_dct3(const double *in, double *out, int nx, int ny, int nz, int inverse) {
    const long V = (long)nx * ny * nz;
    if (out != in) memcpy(out, in, sizeof(double) * V);
    double *Cx = dct_matrix(nx), *Cy = dct_matrix(ny), *Cz = dct_matrix(nz);
    apply_axis(Cz, nz, inverse, out, (long)nx * ny, 1);
    apply_axis(Cy, ny, inverse, out, nx, nz);
    apply_axis(Cx, nx, inverse, out, 1, (long)ny * nz);
    free(Cx); free(Cy); free(Cz);
}

/* Box-Muller normal pair from one Philox draw (23-bit uniforms, same as the CUDA path) */
static inline void normal_pair(uint64_t seed, uint32_t index, uint32_t sweep, uint32_t tag,
                               uint32_t chain, double *z0, double *z1) {
    uint32_t r[4];
    philox_draw(seed, index, sweep, tag, chain, r);
    const double u1 = u01_f24(r[0]), u2 = u01_f24(r[1]);
    const double rr = sqrt(-2.0 * log(u1));
    *z0 = rr * cos(2.0 * PI_D * u2);
    *z1 = rr * sin(2.0 * PI_D * u2);
}

/* NonLinearTransformation.cpp:58-76 (constrain_transformation), :79-126 (sample_transformation),
 * :128-137 (fill_in_data), :151-171 (raw regulariser), :173-188 (update_final_locations),
 * :190-223 (smooth), :344-364 + :433-451 (noise std and draws). */
double orc_smooth(const double *dream, const double *voxel_pos, const double *D,
                  const double gamma[3], double sigma, int nx, int ny, int nz, double *final_out,
                  int add_noise, uint64_t seed, uint32_t sweep, uint32_t chain,
                  const double rho[3], const double eta[3], double *raw_reg) {
    const int N = (nz == 1) ? 2 : 3;
    const long V = (long)nx * ny * nz;
    double *buf = (double *)malloc(sizeof(double) * V);
    double *noise = NULL;
    if (add_noise) {
        noise = (double *)malloc(sizeof(double) * V * 3);
        for (long i = 0; i < V; ++i) {
            double z0, z1, z2, z3;
            normal_pair(seed, (uint32_t)i, sweep, 2u, chain, &z0, &z1);
            normal_pair(seed, (uint32_t)i, sweep, 3u, chain, &z2, &z3);
            noise[i * 3 + 0] = z0; noise[i * 3 + 1] = z1; noise[i * 3 + 2] = z2;
        }
    }
    const double ss2 = sigma * sigma;
    const double rho_p = rho ? rho[0] * rho[1] * rho[2] : 0.0;
    double cost = 0.0, raw = 0.0;
    for (int n = 0; n < N; ++n) {
        for (long i = 0; i < V; ++i) buf[i] = dream[i * N + n] - voxel_pos[i * N + n];
        orc_dct3(buf, buf, nx, ny, nz, 0);
        for (long i = 0; i < V; ++i) {
            double c = buf[i] * (1.0 / (1.0 + gamma[n] * ss2 * D[i]));
            if (add_noise) c += noise[i * 3 + n] * sqrt(ss2 / (1.0 + gamma[n] * ss2 * D[i]));
            if (add_noise && raw_reg) raw += eta[n] * eta[n] * rho_p * D[i] * c * c;
            cost += 0.5 * gamma[n] * D[i] * c * c;
            buf[i] = c;
        }
        orc_dct3(buf, buf, nx, ny, nz, 1);
        for (long i = 0; i < V; ++i) final_out[i * N + n] = buf[i] + voxel_pos[i * N + n];
    }
    if (raw_reg) *raw_reg = raw;
    free(buf);
    free(noise);
    return cost;
}

/* NonLinearTransformation.cpp:280-341 */
void orc_sample_field(const double *field, const double *D, const double gamma[3], double sigma,
                      int nx, int ny, int nz, int n, uint64_t seed, uint32_t sweep0,
                      double *out) {
    const int N = (nz == 1) ? 2 : 3;
    const long V = (long)nx * ny * nz;
    double *zeros = (double *)calloc((size_t)V * N, sizeof(double));
    for (int s = 0; s < n; ++s)
        orc_smooth(field, zeros, D, gamma, sigma, nx, ny, nz, out + (size_t)s * V * N, 1, seed,
                   sweep0 + (uint32_t)s, 0, NULL, NULL, NULL);
    free(zeros);
}

/* NonLinearTransformation.cpp:366-430 (static up_sample): per component, the orthonormal DCT-II on
 * the input grid, its coefficients written into the low-index corner of a zero output spectrum,
 * and the orthonormal DCT-III on the output grid.  AoS [nx][ny][nz][N] -> [nxo][nyo][nzo][N],
 * N = 2 when nzo == 1; every output axis at least as long as the input one. */
void orc_up_sample(const double *in, int nx, int ny, int nz, int nxo, int nyo, int nzo,
                   double *out) {
    const int N = (nzo == 1) ? 2 : 3;
    const long V = (long)nx * ny * nz, Vo = (long)nxo * nyo * nzo;
    double *c = (double *)malloc(sizeof(double) * V);
    double *co = (double *)malloc(sizeof(double) * Vo);
    for (int n = 0; n < N; ++n) {
        for (long p = 0; p < V; ++p) c[p] = in[p * N + n];
        orc_dct3(c, c, nx, ny, nz, 0);
        for (long q = 0; q < Vo; ++q) co[q] = 0.0;
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z)
                    co[((long)x * nyo + y) * nzo + z] = c[((long)x * ny + y) * nz + z];
        orc_dct3(co, co, nxo, nyo, nzo, 1);
        for (long q = 0; q < Vo; ++q) out[q * N + n] = co[q];
    }
    free(c);
    free(co);
}

/* Registration.cpp:122-217 */
int orc_em(double *final_locations, const double *voxel_pos, const int *u, const int *v,
           double *theta, double alpha, const double *D, const double gamma[3], double sigma,
           int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
           double non_zero_voxels, int max_iter, double convergence_th, int update_theta,
           orc_iter_stats *stats) {
    const int N = (nz == 1) ? 2 : 3;
    const long V = (long)nx * ny * nz;
    double *dream = (double *)malloc(sizeof(double) * V * N);
    double *hist = (double *)malloc(sizeof(double) * K * L);
    double mlp_old = 1e100;
    int it = 0;
    while (it < max_iter) {
        const double mll = orc_estep(final_locations, u, v, theta, nx, ny, nz, nxn, nyn, nzn, K, L,
                                     dream, hist, NULL);
        if (update_theta) {
            memcpy(theta, hist, sizeof(double) * K * L);
            orc_theta_map(theta, K, L, alpha);
        }
        const double lpl = orc_dirichlet_cost(theta, K, L, alpha);
        const double lpt = orc_smooth(dream, voxel_pos, D, gamma, sigma, nx, ny, nz,
                                      final_locations, 0, 0, 0, 0, NULL, NULL, NULL);
        const double mlp = mll + lpt + lpl;
        if (stats) {
            stats[it].mll = mll;
            stats[it].log_prior_likelihood = lpl;
            stats[it].log_prior_transformation = lpt;
            stats[it].mlp = mlp;
        }
        ++it;
        if ((mlp_old - mlp) / non_zero_voxels < convergence_th) break;
        mlp_old = mlp;
    }
    free(dream);
    free(hist);
    return it;
}

/* SSDLikelihood.cpp:58-82: log N(u; shift + scale * k, sigmaSq), k = 0 outside the node grid
 * (shiftScale 0: shift 0, scale 1) */
static double ssd_loglik(double uval, int k, const orc_ssd *p) {
    const double adj = p->shift_scale ? uval - p->shift - p->scale * (double)k : uval - (double)k;
    return (adj * adj) / (-2.0 * p->sigma2) - log(sqrt(2.0 * PI_D * p->sigma2));
}

double orc_ssd_estep(const double *d, const int *u, const int *v, const orc_ssd *p, int nx,
                     int ny, int nz, int nxn, int nyn, int nzn, int K, int L, double *dream,
                     double *hist) {
    const int is2D = (nz == 1);
    const int N = is2D ? 2 : 3;
    const long V = (long)nx * ny * nz;
    const int T = orc_get_threads();
    double *hist_t = (double *)calloc((size_t)T * K * L, sizeof(double));
    double mll = 0.0;
#pragma omp parallel num_threads(T) reduction(+ : mll)
    {
#ifdef _OPENMP
        const int tid = omp_get_thread_num();
#else
        const int tid = 0;
#endif
        double *h = hist_t + (size_t)tid * K * L;
#pragma omp for schedule(static)
        for (long i = 0; i < V; ++i) {
            const double *di = d + i * N;
            double bx[4], by[4], bz[4] = {1.0, 1.0, 1.0, 1.0};
            const int ix = spline_setup(di[0], bx), iy = spline_setup(di[1], by);
            const int iz = is2D ? 0 : spline_setup(di[2], bz);
            const int ZZ = is2D ? 1 : 4;
            double lp[64];
            int kb[64], node[64][3];
            int n = 0;
            double mx = -INFINITY;
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b)
                    for (int c = 0; c < ZZ; ++c) {
                        const double w = bx[a] * by[b] * bz[c];
                        if (!(w > 0.0)) continue;  /* the reference's log weight is -1e100 */
                        const int X = ix + a - 1, Y = iy + b - 1, Z = is2D ? 0 : iz + c - 1;
                        const int k = node_bin(v, X, Y, Z, nxn, nyn, nzn);
                        lp[n] = log(bx[a]) + log(by[b]) + (is2D ? 0.0 : log(bz[c])) +
                                ssd_loglik((double)u[i], k, p);
                        kb[n] = k;
                        node[n][0] = X; node[n][1] = Y; node[n][2] = Z;
                        if (lp[n] > mx) mx = lp[n];
                        ++n;
                    }
            double norm = 0.0;
            for (int j = 0; j < n; ++j) norm += exp(lp[j] - mx);
            const double lnorm = log(norm) + mx;
            mll += -lnorm;
            double acc[3] = {0.0, 0.0, 0.0};
            for (int j = 0; j < n; ++j) {
                const double pj = exp(lp[j] - lnorm);
                h[(long)kb[j] * L + u[i]] += pj;
                for (int m = 0; m < N; ++m) acc[m] += pj * (double)node[j][m];
            }
            for (int m = 0; m < N; ++m) dream[i * N + m] = acc[m];
        }
    }
    for (long q = 0; q < (long)K * L; ++q) {
        double s = 0.0;
        for (int t = 0; t < T; ++t) s += hist_t[(size_t)t * K * L + q];
        hist[q] = s;
    }
    free(hist_t);
    return mll;
}

/* update_parameters / update_shift_and_scale / update_sigma (:143-285) from the histogram: the
 * per-node sums of accumulate_info (:111-141) grouped by node bin k (bin 0 also holds the nodes
 * outside the grid, whose contribution is that of a node of value 0); the 2x2 normal equations
 * solved in closed form.  Returns compute_cost (:314-326), the inverse-gamma prior of sigmaSq. */
double orc_ssd_update(const double *hist, int K, int L, orc_ssd *p, int update) {
    if (update) {
        if (!p->shift_scale) {
            double num = 0.0, den = 0.0;
            for (int k = 0; k < K; ++k)
                for (int l = 0; l < L; ++l) {
                    const double h = hist[(long)k * L + l], df = (double)l - (double)k;
                    num += h * df * df;
                    den += h;
                }
            num += p->alpha0 * p->beta0;
            den += p->alpha0;
            p->sigma2 = num / den;
        } else {
            double G[256], S1[256], S2[256];
            double A00 = 0, A01 = 0, A11 = 0, b0 = 0, b1 = 0;
            for (int k = 0; k < K; ++k) {
                G[k] = S1[k] = S2[k] = 0.0;
                for (int l = 0; l < L; ++l) {
                    const double h = hist[(long)k * L + l];
                    G[k] += h;
                    S1[k] += h * (double)l;
                    S2[k] += h * (double)l * (double)l;
                }
                A00 += G[k];
                A01 += G[k] * (double)k;
                A11 += G[k] * (double)k * (double)k;
                b0 += S1[k];
                b1 += S1[k] * (double)k;
            }
            const double det = A00 * A11 - A01 * A01;
            p->shift = (b0 * A11 - A01 * b1) / det;
            p->scale = (A00 * b1 - A01 * b0) / det;
            double num = 0.0, den = 0.0;
            for (int k = 0; k < K; ++k) {
                const double t1 = p->shift + p->scale * (double)k;
                num += S2[k] + -2.0 * S1[k] * t1 + G[k] * (t1 * t1);
                den += G[k];
            }
            num += p->alpha0 * p->beta0;
            den += p->alpha0;
            p->sigma2 = num / den;
        }
    }
    const double a = p->alpha0, b = p->alpha0 * p->beta0, x = p->sigma2;
    return -(a * log(b) - lgamma(a) + (-a - 1.0) * log(x) - b / x);
}

/* SSDLikelihood::sample_parameters (:284-302), update_shift_and_scale and update_sigma with
 * sample = 1 (:167-285), from the sweep's counts hist[k][l] (the drawn node's bin k at voxel bin
 * l).  shiftScale 0: sigmaSq = 1 / g with g ~ Gamma(shape den / 2, scale 2 den / num), the
 * reference's parameterisation as written (num = sum h (l - k)^2 + alpha_0 beta_0, den = sum h +
 * alpha_0).  shiftScale 1: (shift, scale) = A^-1 b + chol(A^-1) z, z two standard normals, then
 * sigmaSq the same way with the drawn shift and scale.  Random numbers: Philox ctr {0, sweep, 6,
 * chain} gives z by Box-Muller on words 0 and 1 (cos, sin); the gamma uses tag 7, index 0.
 * Returns 1 when the gamma draw hit its attempt cap. */
int orc_ssd_sample(const double *hist, int K, int L, orc_ssd *p, uint64_t seed, uint32_t sweep,
                   uint32_t chain) {
    double G[256], S1[256], S2[256];
    for (int k = 0; k < K; ++k) {
        G[k] = S1[k] = S2[k] = 0.0;
        for (int l = 0; l < L; ++l) {
            const double h = hist[(long)k * L + l];
            G[k] += h;
            S1[k] += h * (double)l;
            S2[k] += h * (double)l * (double)l;
        }
    }
    double num = 0.0, den = 0.0;
    if (!p->shift_scale) {
        for (int k = 0; k < K; ++k)
            for (int l = 0; l < L; ++l) {
                const double df = (double)l - (double)k;
                num += hist[(long)k * L + l] * df * df;
            }
        for (int k = 0; k < K; ++k) den += G[k];
    } else {
        double A00 = 0, A01 = 0, A11 = 0, b0 = 0, b1 = 0;
        for (int k = 0; k < K; ++k) {
            A00 += G[k];
            A01 += G[k] * (double)k;
            A11 += G[k] * (double)k * (double)k;
            b0 += S1[k];
            b1 += S1[k] * (double)k;
        }
        const double det = A00 * A11 - A01 * A01;
        const double x0 = (b0 * A11 - A01 * b1) / det, x1 = (A00 * b1 - A01 * b0) / det;
        const double c00 = A11 / det, c01 = -A01 / det, c11 = A00 / det;
        const double l00 = sqrt(c00), l10 = c01 / l00, l11 = sqrt(c11 - l10 * l10);
        uint32_t r[4];
        philox_draw(seed, 0u, sweep, 6u, chain, r);
        const double rad = sqrt(-2.0 * log(u01_d32(r[0]))), ang = 2.0 * PI_D * u01_d32(r[1]);
        const double z0 = rad * cos(ang), z1 = rad * sin(ang);
        p->shift = x0 + l00 * z0;
        p->scale = x1 + l10 * z0 + l11 * z1;
        for (int k = 0; k < K; ++k) {
            const double t1 = p->shift + p->scale * (double)k;
            num += S2[k] + -2.0 * S1[k] * t1 + G[k] * (t1 * t1);
            den += G[k];
        }
    }
    num += p->alpha0 * p->beta0;
    den += p->alpha0;
    int capped = 0;
    const double g = orc_gamma_sample(den * 0.5, seed, 0u, sweep, 7u, chain, &capped) *
                     (2.0 * den / num);
    p->sigma2 = 1.0 / g;
    return capped;
}

/* Registration.cpp:122-217 with the SSD likelihood */
int orc_ssd_em(double *final_locations, const double *voxel_pos, const int *u, const int *v,
               orc_ssd *p, const double *D, const double gamma[3], double sigma, int nx, int ny,
               int nz, int nxn, int nyn, int nzn, int K, int L, double non_zero_voxels,
               int max_iter, double convergence_th, int update, orc_iter_stats *stats) {
    const int N = (nz == 1) ? 2 : 3;
    const long V = (long)nx * ny * nz;
    double *dream = (double *)malloc(sizeof(double) * V * N);
    double *hist = (double *)malloc(sizeof(double) * K * L);
    double mlp_old = 1e100;
    int it = 0;
    while (it < max_iter) {
        const double mll = orc_ssd_estep(final_locations, u, v, p, nx, ny, nz, nxn, nyn, nzn, K,
                                         L, dream, hist);
        const double lpl = orc_ssd_update(hist, K, L, p, update);
        const double lpt = orc_smooth(dream, voxel_pos, D, gamma, sigma, nx, ny, nz,
                                      final_locations, 0, 0, 0, 0, NULL, NULL, NULL);
        const double mlp = mll + lpt + lpl;
        if (stats) {
            stats[it].mll = mll;
            stats[it].log_prior_likelihood = lpl;
            stats[it].log_prior_transformation = lpt;
            stats[it].mlp = mlp;
        }
        ++it;
        if ((mlp_old - mlp) / non_zero_voxels < convergence_th) break;
        mlp_old = mlp;
    }
    free(dream);
    free(hist);
    return it;
}

/* Registration.cpp:515-642 with NonLinearTransformation.cpp:79-126 for block 3 */
int orc_sampler(double *final_locations, double *dream, const double *voxel_pos, const int *u,
                const int *v, double *theta, double alpha, const double *D, double gamma[3],
                double sigma, const double rho[3], const double eta[3],
                int nx, int ny, int nz, int nxn, int nyn, int nzn, int K, int L,
                uint64_t seed, uint32_t chain, int N_b, int N_s, int sample_gamma,
                int sample_gamma_every, int sample_posteriors, int sample_likelihood_parameters,
                int sample_transformation_parameters, double *mean_out, double *cov_out) {
    const int N = (nz == 1) ? 2 : 3;
    const long V = (long)nx * ny * nz;
    double *hist = (double *)calloc((size_t)K * L, sizeof(double));
    double *M2 = (double *)calloc((size_t)V * N * N, sizeof(double));
    memset(mean_out, 0, sizeof(double) * V * N);
    const double alpha_0 = 1.0, beta_0 = 10000.0; /* NonLinearTransformation.cpp:41-42 */
    int capped = 0;
    for (int sweep = 0; sweep < N_b + N_s; ++sweep) {
        if (sample_posteriors)
            orc_estep_sample(final_locations, u, v, theta, nx, ny, nz, nxn, nyn, nzn, K, L, seed,
                             (uint32_t)sweep, chain, dream, hist);
        if (sample_likelihood_parameters) {
            memcpy(theta, hist, sizeof(double) * K * L);
            capped += orc_dirichlet_sample(theta, K, L, alpha, seed, (uint32_t)sweep, chain);
        }
        if (sample_transformation_parameters) {
            const int sg = sample_gamma && (sweep % sample_gamma_every == 0);
            double raw = 0.0;
            orc_smooth(dream, voxel_pos, D, gamma, sigma, nx, ny, nz, final_locations, 1, seed,
                       (uint32_t)sweep, chain, rho, eta, sg ? &raw : NULL);
            if (sg) {
                const double a_post = alpha_0 + 0.5 * (double)(N * V);
                const double b_post = beta_0 + 0.5 * (double)V * raw;
                int c = 0;
                const double nu = orc_gamma_sample(a_post, seed, 0u, (uint32_t)sweep, 5u, chain, &c) /
                                  b_post;
                capped += c;
                const double rp = rho[0] * rho[1] * rho[2];
                for (int n = 0; n < 3; ++n) gamma[n] = nu * rp * eta[n] * eta[n] * (double)V;
            }
        }
        if (sweep >= N_b) {
            const double inv_n = 1.0 / ((double)(sweep - N_b) + 1.0);
            for (long i = 0; i < V; ++i) {
                double d1[3], d2[3];
                for (int n = 0; n < N; ++n) {
                    const double val = final_locations[i * N + n];
                    const double m_old = mean_out[i * N + n];
                    d1[n] = val - m_old;
                    const double m_new = m_old + d1[n] * inv_n;
                    mean_out[i * N + n] = m_new;
                    d2[n] = val - m_new;
                }
                for (int r = 0; r < N; ++r)
                    for (int c = 0; c < N; ++c) M2[i * N * N + r * N + c] += d1[r] * d2[c];
            }
        }
    }
    const double inv = 1.0 / (double)(N_s - 1);
    for (long q = 0; q < V * N * N; ++q) cov_out[q] = M2[q] * inv;
    free(hist);
    free(M2);
    return capped;
}

/* ------------------------------------------------------------------------------------------ */
/* Jacobian determinants                                                                       */
/* ------------------------------------------------------------------------------------------ */
/* cofactor expansion along the first row, the grouping the reference writes out
 * (BINDER/src/cpu/utils.cpp:156-160 and topology_correction_3D.cpp:286-288) */
static inline double det3(double a00, double a01, double a02, double a10, double a11, double a12,
                          double a20, double a21, double a22) {
    return a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) +
           a02 * (a10 * a21 - a11 * a20);
}

/* BINDER/src/cpu/utils.cpp:100-345: mean over the valid ones of the 8 one-sided corner
 * determinants at every voxel; corners visited in the order fff, bff, fbf, ffb, bbf, bfb, fbb,
 * bbb (f = forward difference along that axis, b = backward). */
void orc_jacobian3d(const double *f, int nx, int ny, int nz, double vx, double vy, double vz,
                    double *J) {
    static const int dirs[8][3] = {{1, 1, 1},  {-1, 1, 1},  {1, -1, 1},  {1, 1, -1},
                                   {-1, -1, 1}, {-1, 1, -1}, {1, -1, -1}, {-1, -1, -1}};
    const double vol = 1.0 / (vx * vy * vz);
    const int T = orc_get_threads();
#pragma omp parallel for num_threads(T) schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const long p = ((long)x * ny + y) * nz + z;
                const double *w0 = f + p * 3;
                double tot = 0.0;
                int valid = 0;
                for (int c = 0; c < 8; ++c) {
                    const int sx = dirs[c][0], sy = dirs[c][1], sz = dirs[c][2];
                    if ((sx > 0 && x >= nx - 1) || (sx < 0 && x <= 0)) continue;
                    if ((sy > 0 && y >= ny - 1) || (sy < 0 && y <= 0)) continue;
                    if ((sz > 0 && z >= nz - 1) || (sz < 0 && z <= 0)) continue;
                    const double *px = f + (p + (long)sx * ny * nz) * 3;
                    const double *py = f + (p + (long)sy * nz) * 3;
                    const double *pz = f + (p + sz) * 3;
                    double col[3][3]; /* col[axis][component] */
                    for (int m = 0; m < 3; ++m) {
                        col[0][m] = sx > 0 ? px[m] - w0[m] : w0[m] - px[m];
                        col[1][m] = sy > 0 ? py[m] - w0[m] : w0[m] - py[m];
                        col[2][m] = sz > 0 ? pz[m] - w0[m] : w0[m] - pz[m];
                    }
                    const double Jc = det3(col[0][0], col[1][0], col[2][0], col[0][1], col[1][1],
                                           col[2][1], col[0][2], col[1][2], col[2][2]) * vol;
                    tot += Jc;
                    valid++;
                }
                J[p] = valid > 0 ? tot / valid : 1.0;
            }
}

/* BINDER/src/cpu/utils.cpp:10-98: mean over the valid ones of the 4 one-sided corner
 * determinants (ff, bf, fb, bb) */
void orc_jacobian2d(const double *f, int nx, int ny, double vx, double vy, double *J) {
    static const int dirs[4][2] = {{1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
    const double vol = 1.0 / (vx * vy);
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            const long p = (long)x * ny + y;
            const double *w0 = f + p * 2;
            double tot = 0.0;
            int valid = 0;
            for (int c = 0; c < 4; ++c) {
                const int sx = dirs[c][0], sy = dirs[c][1];
                if ((sx > 0 && x >= nx - 1) || (sx < 0 && x <= 0)) continue;
                if ((sy > 0 && y >= ny - 1) || (sy < 0 && y <= 0)) continue;
                const double *px = f + (p + (long)sx * ny) * 2;
                const double *py = f + (p + sy) * 2;
                const double ax0 = sx > 0 ? px[0] - w0[0] : w0[0] - px[0];
                const double ax1 = sx > 0 ? px[1] - w0[1] : w0[1] - px[1];
                const double ay0 = sy > 0 ? py[0] - w0[0] : w0[0] - py[0];
                const double ay1 = sy > 0 ? py[1] - w0[1] : w0[1] - py[1];
                tot += (ax0 * ay1 - ay0 * ax1) * vol;
                valid++;
            }
            J[p] = valid > 0 ? tot / valid : 1.0;
        }
}

/* ------------------------------------------------------------------------------------------ */
/* topology correction (BINDER/src/cpu/topology_correction_3D.cpp)                             */
/* ------------------------------------------------------------------------------------------ */
/* :488-607: the 8 corner Jacobians of every cell (x..x+1, y..y+1, z..z+1), stored in the order
 * of the cell vertices 000, 100, 010, 001, 011, 101, 110, 111; each uses the three cell edges
 * through its vertex (hi - lo). */
void orc_corner_jacobians3d(const double *pos, int nx, int ny, int nz, const double vs[3],
                            double e1, double e2, double *Jc, int *n_below, int *n_above) {
    static const int vert[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                   {0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
    const double vol = 1.0 / (vs[0] * vs[1] * vs[2]);
    long nb = 0, na = 0;
    const int T = orc_get_threads();
#pragma omp parallel for num_threads(T) schedule(static) reduction(+ : nb, na)
    for (int x = 0; x < nx - 1; ++x)
        for (int y = 0; y < ny - 1; ++y)
            for (int z = 0; z < nz - 1; ++z) {
                const long cell = ((long)x * (ny - 1) + y) * (nz - 1) + z;
                for (int c = 0; c < 8; ++c) {
                    const int cx = vert[c][0], cy = vert[c][1], cz = vert[c][2];
                    const double *w = pos + (((long)(x + cx) * ny + (y + cy)) * nz + (z + cz)) * 3;
                    /* neighbours across each edge through the vertex */
                    const double *wx = pos + (((long)(x + 1 - cx) * ny + (y + cy)) * nz + (z + cz)) * 3;
                    const double *wy = pos + (((long)(x + cx) * ny + (y + 1 - cy)) * nz + (z + cz)) * 3;
                    const double *wz = pos + (((long)(x + cx) * ny + (y + cy)) * nz + (z + 1 - cz)) * 3;
                    double col[3][3];
                    for (int m = 0; m < 3; ++m) {
                        col[0][m] = cx ? w[m] - wx[m] : wx[m] - w[m];
                        col[1][m] = cy ? w[m] - wy[m] : wy[m] - w[m];
                        col[2][m] = cz ? w[m] - wz[m] : wz[m] - w[m];
                    }
                    double j = det3(col[0][0], col[1][0], col[2][0], col[0][1], col[1][1], col[2][1],
                                    col[0][2], col[1][2], col[2][2]);
                    j *= vol;
                    Jc[cell * 8 + c] = j;
                    if (j < e1) nb++;
                    if (j > e2) na++;
                }
            }
    if (n_below) *n_below = (int)nb;
    if (n_above) *n_above = (int)na;
}

/* :172-245: forward differences with periodic wrap, grad[p][n1*3+n2] = d pos_n1 / d axis_n2 / vs[n1] */
void orc_gradients3d(const double *pos, int nx, int ny, int nz, const double vs[3], double *g) {
    const int T = orc_get_threads();
#pragma omp parallel for num_threads(T) schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const long p = ((long)x * ny + y) * nz + z;
                const int x2 = (x + 1 > nx - 1) ? x + 1 - nx : x + 1;
                const int y2 = (y + 1 > ny - 1) ? y + 1 - ny : y + 1;
                const int z2 = (z + 1 > nz - 1) ? z + 1 - nz : z + 1;
                const long px = ((long)x2 * ny + y) * nz + z;
                const long py = ((long)x * ny + y2) * nz + z;
                const long pz = ((long)x * ny + y) * nz + z2;
                for (int n1 = 0; n1 < 3; ++n1) {
                    g[p * 9 + n1 * 3 + 0] = (pos[px * 3 + n1] - pos[p * 3 + n1]) / vs[n1];
                    g[p * 9 + n1 * 3 + 1] = (pos[py * 3 + n1] - pos[p * 3 + n1]) / vs[n1];
                    g[p * 9 + n1 * 3 + 2] = (pos[pz * 3 + n1] - pos[p * 3 + n1]) / vs[n1];
                }
            }
}

/* :247-332 and :452-486: in lexicographic cell order, every flagged corner's gradient matrix is
 * blended toward the identity in steps of 0.1 until its determinant lies in [e1, e2], then one
 * more step is applied and written back.  The blending loop is capped at 11 steps (alpha = 1
 * gives the identity); returns the number of corners that hit the cap. */
int orc_limit_gradients3d(double *g, const double *Jc, int nx, int ny, int nz, double e1,
                          double e2) {
    static const int vert[8][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1},
                                   {0, 1, 1}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
    int capped = 0;
    for (int x = 0; x < nx - 1; ++x)
        for (int y = 0; y < ny - 1; ++y)
            for (int z = 0; z < nz - 1; ++z)
                for (int c = 0; c < 8; ++c) {
                    const long cell = ((long)x * (ny - 1) + y) * (nz - 1) + z;
                    const double jv = Jc[cell * 8 + c];
                    if (!(jv < e1 || jv > e2)) continue;
                    /* column n2 is the forward difference stored at the vertex minus its n2 bit */
                    long gp[3];
                    for (int n2 = 0; n2 < 3; ++n2) {
                        int o[3] = {vert[c][0], vert[c][1], vert[c][2]};
                        o[n2] = 0;
                        gp[n2] = ((long)(x + o[0]) * ny + (y + o[1])) * nz + (z + o[2]);
                    }
                    double J[3][3];
                    for (int n1 = 0; n1 < 3; ++n1)
                        for (int n2 = 0; n2 < 3; ++n2) J[n1][n2] = g[gp[n2] * 9 + n1 * 3 + n2];
                    double alpha = 0.0;
                    double det = det3(J[0][0], J[0][1], J[0][2], J[1][0], J[1][1], J[1][2], J[2][0],
                                      J[2][1], J[2][2]);
                    int steps = 0;
                    while (det > e2 || det < e1) {
                        if (++steps > 11) { capped++; break; }
                        alpha += 0.1;
                        if (alpha > 1.0) alpha = 1.0;
                        double Jn[3][3];
                        for (int n1 = 0; n1 < 3; ++n1)
                            for (int n2 = 0; n2 < 3; ++n2)
                                Jn[n1][n2] = (1 - alpha) * J[n1][n2] + alpha * (n1 == n2 ? 1.0 : 0.0);
                        det = det3(Jn[0][0], Jn[0][1], Jn[0][2], Jn[1][0], Jn[1][1], Jn[1][2],
                                   Jn[2][0], Jn[2][1], Jn[2][2]);
                    }
                    alpha += 0.1;
                    if (alpha > 1.0) alpha = 1.0;
                    for (int n1 = 0; n1 < 3; ++n1)
                        for (int n2 = 0; n2 < 3; ++n2)
                            g[gp[n2] * 9 + n1 * 3 + n2] =
                                (1 - alpha) * J[n1][n2] + alpha * (n1 == n2 ? 1.0 : 0.0);
                }
    return capped;
}

/* complex DFT along one axis (FFTW sign convention: forward e^{-2 pi i jk/n}, unnormalised) */
static void dft_axis(double *re, double *im, int n, long outer, long s, int sign) {
    double *cs = (double *)malloc(sizeof(double) * n), *sn = (double *)malloc(sizeof(double) * n);
    for (int m = 0; m < n; ++m) {
        cs[m] = cos(2.0 * PI_D * m / n);
        sn[m] = sin(2.0 * PI_D * m / n);
    }
    const int T = orc_get_threads();
#pragma omp parallel num_threads(T)
    {
        double *ir = (double *)malloc(sizeof(double) * n), *ii = (double *)malloc(sizeof(double) * n);
#pragma omp for schedule(static)
        for (long o = 0; o < outer * s; ++o) {
            const long b = (o / s) * (long)n * s + (o % s);
            for (int j = 0; j < n; ++j) { ir[j] = re[b + j * s]; ii[j] = im[b + j * s]; }
            for (int k = 0; k < n; ++k) {
                double ar = 0.0, ai = 0.0;
                for (int j = 0; j < n; ++j) {
                    const int m = (int)(((long)j * k) % n);
                    const double c = cs[m], sgn_s = sign * sn[m];
                    ar += ir[j] * c - ii[j] * sgn_s;
                    ai += ir[j] * sgn_s + ii[j] * c;
                }
                re[b + k * s] = ar;
                im[b + k * s] = ai;
            }
        }
        free(ir); free(ii);
    }
    free(cs); free(sn);
}

static void dft3(double *re, double *im, int nx, int ny, int nz, int sign) {
    dft_axis(re, im, nz, (long)nx * ny, 1, sign);
    dft_axis(re, im, ny, nx, nz, sign);
    dft_axis(re, im, nx, 1, (long)ny * nz, sign);
}

/* :361-449: periodic Poisson integration of each component's gradient field, then rescale by
 * the voxel size and restore the mean */
void orc_integrate3d(double *pos, const double *g, int nx, int ny, int nz, const double vs[3],
                     const double mean[3]) {
    const long V = (long)nx * ny * nz;
    double *re[3], *im[3];
    for (int a = 0; a < 3; ++a) {
        re[a] = (double *)malloc(sizeof(double) * V);
        im[a] = (double *)malloc(sizeof(double) * V);
    }
    for (int n = 0; n < 3; ++n) {
        for (int a = 0; a < 3; ++a) {
            for (long p = 0; p < V; ++p) { re[a][p] = g[p * 9 + n * 3 + a]; im[a][p] = 0.0; }
            dft3(re[a], im[a], nx, ny, nz, -1);
        }
        for (int x = 0; x < nx; ++x) {
            const double cx = cos(2.0 * PI_D * x / (nx * 1.0)), sx = sin(2.0 * PI_D * x / (nx * 1.0));
            for (int y = 0; y < ny; ++y) {
                const double cy = cos(2.0 * PI_D * y / (ny * 1.0)), sy = sin(2.0 * PI_D * y / (ny * 1.0));
                for (int z = 0; z < nz; ++z) {
                    const double cz = cos(2.0 * PI_D * z / (nz * 1.0)), sz = sin(2.0 * PI_D * z / (nz * 1.0));
                    const long p = ((long)x * ny + y) * nz + z;
                    const double nrm = 6.0 - 2.0 * cz - 2.0 * cx - 2.0 * cy;
                    if (fabs(nrm) > 1e-10) {
                        const double dr = re[0][p] * (cx - 1) + im[0][p] * sx + re[1][p] * (cy - 1) +
                                          im[1][p] * sy + re[2][p] * (cz - 1) + im[2][p] * sz;
                        const double di = im[0][p] * (cx - 1) - re[0][p] * sx + im[1][p] * (cy - 1) -
                                          re[1][p] * sy + im[2][p] * (cz - 1) - re[2][p] * sz;
                        re[0][p] = dr / nrm;
                        im[0][p] = di / nrm;
                    } else {
                        re[0][p] = 0.0;
                        im[0][p] = 0.0;
                    }
                }
            }
        }
        dft3(re[0], im[0], nx, ny, nz, +1);
        for (long p = 0; p < V; ++p) pos[p * 3 + n] = re[0][p] / (nx * ny * nz * 1.0);
    }
    for (long p = 0; p < V; ++p)
        for (int n = 0; n < 3; ++n) {
            pos[p * 3 + n] *= vs[n];
            pos[p * 3 + n] += mean[n];
        }
    for (int a = 0; a < 3; ++a) { free(re[a]); free(im[a]); }
}

static void minmax(const double *J, long V, double *mn, double *mx) {
    double a = J[0], b = J[0];
    for (long i = 1; i < V; ++i) {
        if (J[i] < a) a = J[i];
        if (J[i] > b) b = J[i];
    }
    *mn = a;
    *mx = b;
}

/* :17-143 */
int orc_topology3d(double *field, double e1, double e2, int max_outer, int max_inner,
                   const double vs[3], int nx, int ny, int nz) {
    const long V = (long)nx * ny * nz;
    for (long p = 0; p < V; ++p)
        for (int n = 0; n < 3; ++n) field[p * 3 + n] *= vs[n];
    double *J = (double *)malloc(sizeof(double) * V);
    orc_jacobian3d(field, nx, ny, nz, vs[0], vs[1], vs[2], J);
    double jmin, jmax;
    minmax(J, V, &jmin, &jmax);
    int outer = 0;
    if (!(jmin >= e1 && jmax <= e2)) {
        const long cells = (long)(nx - 1) * (ny - 1) * (nz - 1);
        double *Jc = (double *)malloc(sizeof(double) * (cells > 0 ? cells : 1) * 8);
        double *g = (double *)malloc(sizeof(double) * V * 9);
        while ((jmin < e1 || jmax > e2) && outer < max_outer) {
            int nb = 0, na = 0;
            orc_corner_jacobians3d(field, nx, ny, nz, vs, e1, e2, Jc, &nb, &na);
            int inner = 0;
            while ((nb > 0 || na > 0) && inner < max_inner) {
                orc_gradients3d(field, nx, ny, nz, vs, g);
                orc_limit_gradients3d(g, Jc, nx, ny, nz, e1, e2);
                double mean[3] = {0.0, 0.0, 0.0};
                for (long p = 0; p < V; ++p)
                    for (int n = 0; n < 3; ++n) mean[n] += field[p * 3 + n];
                for (int n = 0; n < 3; ++n) mean[n] = mean[n] / (nx * ny * nz);
                orc_integrate3d(field, g, nx, ny, nz, vs, mean);
                orc_corner_jacobians3d(field, nx, ny, nz, vs, e1, e2, Jc, &nb, &na);
                inner++;
            }
            orc_jacobian3d(field, nx, ny, nz, vs[0], vs[1], vs[2], J);
            minmax(J, V, &jmin, &jmax);
            outer++;
        }
        free(Jc);
        free(g);
    }
    for (long p = 0; p < V; ++p)
        for (int n = 0; n < 3; ++n) field[p * 3 + n] /= vs[n];
    free(J);
    return outer;
}

/* ------------------------------------------------------------------------------------------ */
/* 2D topology correction (BINDER/src/cpu/topology_correction_2D.cpp)                          */
/* ------------------------------------------------------------------------------------------ */
/* :165-207: 4 corner Jacobians per cell (x..x+1, y..y+1), in the vertex order 00, 10, 01, 11
 * (the reference's Jff, Jbf, Jfb, Jbb).  Corner (vx, vy) uses the x edge at y + vy and the y edge
 * at x + vx (hi - lo each): det = ex_x * ey_y - ey_x * ex_y, then times 1 / (vs0 vs1).  The
 * counters count CELLS with a corner below e1 / above e2, as the reference's do. */
void orc_corner_jacobians2d(const double *pos, int nx, int ny, const double vs[2], double e1,
                            double e2, double *Jc, int *n_below, int *n_above) {
    const double vol = 1.0 / (vs[0] * vs[1]);
    long nb = 0, na = 0;
    for (int x = 0; x < nx - 1; ++x)
        for (int y = 0; y < ny - 1; ++y) {
            const long cell = (long)x * (ny - 1) + y;
            int lo = 0, hi = 0;
            for (int c = 0; c < 4; ++c) {
                const int vx = c & 1, vy = c >> 1;
                const double *a0 = pos + ((long)x * ny + (y + vy)) * 2;        /* x edge, low  */
                const double *a1 = pos + ((long)(x + 1) * ny + (y + vy)) * 2;  /* x edge, high */
                const double *b0 = pos + ((long)(x + vx) * ny + y) * 2;        /* y edge, low  */
                const double *b1 = pos + ((long)(x + vx) * ny + (y + 1)) * 2;  /* y edge, high */
                const double j = ((a1[0] - a0[0]) * (b1[1] - b0[1]) -
                                  (b1[0] - b0[0]) * (a1[1] - a0[1])) * vol;
                Jc[cell * 4 + c] = j;
                lo |= j < e1;
                hi |= j > e2;
            }
            nb += lo;
            na += hi;
        }
    if (n_below) *n_below = (int)nb;
    if (n_above) *n_above = (int)na;
}

/* :209-246: periodic forward differences, g[p*4 + n1*2 + n2] = d pos_n1 / d axis_n2 / vs[n1] */
void orc_gradients2d(const double *pos, int nx, int ny, const double vs[2], double *g) {
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y) {
            const long p = (long)x * ny + y;
            const long px = (long)((x + 1 > nx - 1) ? x + 1 - nx : x + 1) * ny + y;
            const long py = (long)x * ny + ((y + 1 > ny - 1) ? y + 1 - ny : y + 1);
            for (int n1 = 0; n1 < 2; ++n1) {
                g[p * 4 + n1 * 2 + 0] = (pos[px * 2 + n1] - pos[p * 2 + n1]) / vs[n1];
                g[p * 4 + n1 * 2 + 1] = (pos[py * 2 + n1] - pos[p * 2 + n1]) / vs[n1];
            }
        }
}

/* :248-313 and :390-406: the 3D limiter's rule on 2x2 gradient matrices -- lexicographic cell
 * order, corners in order, column n2 read at the corner's vertex with its n2 bit cleared, blended
 * toward the identity in 0.1 steps (capped at 11; returns the corners that hit the cap). */
int orc_limit_gradients2d(double *g, const double *Jc, int nx, int ny, double e1, double e2) {
    int capped = 0;
    for (int x = 0; x < nx - 1; ++x)
        for (int y = 0; y < ny - 1; ++y)
            for (int c = 0; c < 4; ++c) {
                const double jv = Jc[((long)x * (ny - 1) + y) * 4 + c];
                if (!(jv < e1 || jv > e2)) continue;
                const int vx = c & 1, vy = c >> 1;
                const long gp[2] = {(long)x * ny + (y + vy), (long)(x + vx) * ny + y};
                double J[2][2];
                for (int n1 = 0; n1 < 2; ++n1)
                    for (int n2 = 0; n2 < 2; ++n2) J[n1][n2] = g[gp[n2] * 4 + n1 * 2 + n2];
                double alpha = 0.0;
                double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                int steps = 0;
                while (det > e2 || det < e1) {
                    if (++steps > 11) { capped++; break; }
                    alpha += 0.1;
                    if (alpha > 1.0) alpha = 1.0;
                    double Jn[2][2];
                    for (int n1 = 0; n1 < 2; ++n1)
                        for (int n2 = 0; n2 < 2; ++n2)
                            Jn[n1][n2] = (1 - alpha) * J[n1][n2] + alpha * (n1 == n2 ? 1.0 : 0.0);
                    det = Jn[0][0] * Jn[1][1] - Jn[0][1] * Jn[1][0];
                }
                alpha += 0.1;
                if (alpha > 1.0) alpha = 1.0;
                for (int n1 = 0; n1 < 2; ++n1)
                    for (int n2 = 0; n2 < 2; ++n2)
                        g[gp[n2] * 4 + n1 * 2 + n2] =
                            (1 - alpha) * J[n1][n2] + alpha * (n1 == n2 ? 1.0 : 0.0);
            }
    return capped;
}

/* :315-388: per component, the gradient spectra X, Y combine to
 * ((e^{-i tx} - 1) X + (e^{-i ty} - 1) Y) / (4 - 2 cos ty - 2 cos tx) (zero where that is
 * <= 1e-10), inverse transformed, divided by nx ny, scaled by the voxel size, plus the mean */
void orc_integrate2d(double *pos, const double *g, int nx, int ny, const double vs[2],
                     const double mean[2]) {
    const long V = (long)nx * ny;
    double *xr = (double *)malloc(sizeof(double) * V), *xi = (double *)malloc(sizeof(double) * V);
    double *yr = (double *)malloc(sizeof(double) * V), *yi = (double *)malloc(sizeof(double) * V);
    for (int n = 0; n < 2; ++n) {
        for (long p = 0; p < V; ++p) {
            xr[p] = g[p * 4 + n * 2 + 0]; xi[p] = 0.0;
            yr[p] = g[p * 4 + n * 2 + 1]; yi[p] = 0.0;
        }
        dft3(xr, xi, nx, ny, 1, -1);
        dft3(yr, yi, nx, ny, 1, -1);
        for (int x = 0; x < nx; ++x) {
            const double cx = cos(2.0 * PI_D * x / nx), sx = sin(2.0 * PI_D * x / nx);
            for (int y = 0; y < ny; ++y) {
                const double cy = cos(2.0 * PI_D * y / ny), sy = sin(2.0 * PI_D * y / ny);
                const long p = (long)x * ny + y;
                const double nrm = 4.0 - 2.0 * cy - 2.0 * cx;
                if (nrm > 1e-10) {
                    const double r = (xr[p] * (cx - 1.0) + xi[p] * sx + yr[p] * (cy - 1.0) + yi[p] * sy) / nrm;
                    const double i = (xi[p] * (cx - 1.0) - xr[p] * sx + yi[p] * (cy - 1.0) - yr[p] * sy) / nrm;
                    xr[p] = r;
                    xi[p] = i;
                } else {
                    xr[p] = 0.0;
                    xi[p] = 0.0;
                }
            }
        }
        dft3(xr, xi, nx, ny, 1, +1);
        for (long p = 0; p < V; ++p)
            pos[p * 2 + n] = xr[p] * (1.0 / (nx * ny)) * vs[n] + mean[n];
    }
    free(xr); free(xi); free(yr); free(yi);
}

/* :17-163 on an AoS [nx][ny][2] field in grid units (in place); returns the outer iterations */
int orc_topology2d(double *field, double e1, double e2, int max_outer, int max_inner,
                   const double vs[2], int nx, int ny) {
    const long V = (long)nx * ny;
    for (long p = 0; p < V; ++p)
        for (int n = 0; n < 2; ++n) field[p * 2 + n] *= vs[n];
    double *J = (double *)malloc(sizeof(double) * V);
    orc_jacobian2d(field, nx, ny, vs[0], vs[1], J);
    double jmin, jmax;
    minmax(J, V, &jmin, &jmax);
    int outer = 0;
    if (!(jmin >= e1 && jmax <= e2)) {
        const long cells = (long)(nx - 1) * (ny - 1);
        double *Jc = (double *)malloc(sizeof(double) * (cells > 0 ? cells : 1) * 4);
        double *g = (double *)malloc(sizeof(double) * V * 4);
        while ((jmin < e1 || jmax > e2) && outer < max_outer) {
            int nb = 0, na = 0;
            orc_corner_jacobians2d(field, nx, ny, vs, e1, e2, Jc, &nb, &na);
            int inner = 0;
            while ((nb > 0 || na > 0) && inner < max_inner) {
                orc_gradients2d(field, nx, ny, vs, g);
                orc_limit_gradients2d(g, Jc, nx, ny, e1, e2);
                double mean[2] = {0.0, 0.0};
                for (long p = 0; p < V; ++p)
                    for (int n = 0; n < 2; ++n) mean[n] += field[p * 2 + n];
                for (int n = 0; n < 2; ++n) mean[n] = mean[n] / (nx * ny);
                orc_integrate2d(field, g, nx, ny, vs, mean);
                orc_corner_jacobians2d(field, nx, ny, vs, e1, e2, Jc, &nb, &na);
                inner++;
            }
            orc_jacobian2d(field, nx, ny, vs[0], vs[1], J);
            minmax(J, V, &jmin, &jmax);
            outer++;
        }
        free(Jc);
        free(g);
    }
    for (long p = 0; p < V; ++p)
        for (int n = 0; n < 2; ++n) field[p * 2 + n] /= vs[n];
    free(J);
    return outer;
}

/* MI of the joint distribution given by a (soft) joint histogram */
double orc_mutual_information(const double *h, int K, int L) {
    double tot = 0.0;
    for (long q = 0; q < (long)K * L; ++q) tot += h[q];
    if (!(tot > 0.0)) return 0.0;
    double *pk = (double *)calloc(K, sizeof(double)), *pl = (double *)calloc(L, sizeof(double));
    for (int k = 0; k < K; ++k)
        for (int l = 0; l < L; ++l) {
            pk[k] += h[k * L + l] / tot;
            pl[l] += h[k * L + l] / tot;
        }
    double mi = 0.0;
    for (int k = 0; k < K; ++k)
        for (int l = 0; l < L; ++l) {
            const double p = h[k * L + l] / tot;
            if (p > 0.0) mi += p * log(p / (pk[k] * pl[l]));
        }
    free(pk);
    free(pl);
    return mi;
}

/* ---- SSD filter likelihood: BINDER/src/cpu/SSDLikelihoodFilter.cpp ------------------------- */

/* the predicted value of channel m at node j: sum_f coeff[m][f] nodes[j][f] (reg_across_features
 * 0, nodes [Vn][F]) or nodes[j][m] (1, nodes [Vn][M]); 0 outside the grid */
static double ssdf_pred(const orc_ssdf *p, const double *nodes, long node, int m) {
    if (node < 0) return 0.0;
    if (p->rfa) return nodes[node * p->M + m];
    double t = 0.0;
    for (int f = 0; f < p->F; ++f) t += p->coeff[m * p->F + f] * nodes[node * p->F + f];
    return t;
}

/* compute_log_likelihood (:123-158) */
double orc_ssdf_loglik(const orc_ssdf *p, const double *nodes, const double *voxels, int nxn,
                       int nyn, int nzn, long voxel, int x, int y, int z) {
    const int outside = x < 0 || y < 0 || z < 0 || x >= nxn || y >= nyn || z >= nzn;
    const long node = outside ? -1 : ((long)x * nyn + y) * nzn + z;
    double ll = 0.0;
    for (int m = 0; m < p->M; ++m) {
        double t = voxels[voxel * p->M + m];
        if (!outside) t -= ssdf_pred(p, nodes, node, m);
        ll += (t * t) / (-2.0 * p->sigma[m]) - 0.5 * log(2.0 * PI_D * p->sigma[m]);
    }
    return ll;
}

/* The log-space E-step (Registration.cpp:331-470) with the filter likelihood and the
 * accumulators of accumulate_info (:160-198): gamma [Vn], s1 [M][Vn], s2 [M][Vn] per node;
 * outside [1 + 2M] = (gamma, s1[M], s2[M]) of the nodes outside the grid.  Serial. */
double orc_ssdf_estep(const double *d, const double *nodes, const double *voxels,
                      const orc_ssdf *p, int nx, int ny, int nz, int nxn, int nyn, int nzn,
                      double *dream, double *gamma, double *s1, double *s2, double *outside) {
    const int is2D = (nz == 1);
    const int N = is2D ? 2 : 3;
    const long V = (long)nx * ny * nz, Vn = (long)nxn * nyn * nzn;
    const int M = p->M;
    memset(gamma, 0, sizeof(double) * Vn);
    memset(s1, 0, sizeof(double) * M * Vn);
    memset(s2, 0, sizeof(double) * M * Vn);
    memset(outside, 0, sizeof(double) * (1 + 2 * M));
    double mll = 0.0;
    for (long i = 0; i < V; ++i) {
        const double *di = d + i * N;
        double bx[4], by[4], bz[4] = {1.0, 1.0, 1.0, 1.0};
        const int ix = spline_setup(di[0], bx), iy = spline_setup(di[1], by);
        const int iz = is2D ? 0 : spline_setup(di[2], bz);
        const int ZZ = is2D ? 1 : 4;
        double lp[64];
        int node[64][3];
        int n = 0;
        double mx = -INFINITY;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b)
                for (int c = 0; c < ZZ; ++c) {
                    const double w = bx[a] * by[b] * bz[c];
                    if (!(w > 0.0)) continue;  /* a zero tap has no posterior mass */
                    const int X = ix + a - 1, Y = iy + b - 1, Z = is2D ? 0 : iz + c - 1;
                    lp[n] = log(bx[a]) + log(by[b]) + (is2D ? 0.0 : log(bz[c])) +
                            orc_ssdf_loglik(p, nodes, voxels, nxn, nyn, nzn, i, X, Y, Z);
                    node[n][0] = X; node[n][1] = Y; node[n][2] = Z;
                    if (lp[n] > mx) mx = lp[n];
                    ++n;
                }
        double norm = 0.0;
        for (int j = 0; j < n; ++j) norm += exp(lp[j] - mx);
        const double lnorm = log(norm) + mx;
        mll += -lnorm;
        double acc[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < n; ++j) {
            const double pj = exp(lp[j] - lnorm);
            const int X = node[j][0], Y = node[j][1], Z = node[j][2];
            const int out = X < 0 || Y < 0 || Z < 0 || X >= nxn || Y >= nyn || Z >= nzn;
            if (!out) {
                const long nj = ((long)X * nyn + Y) * nzn + Z;
                gamma[nj] += pj;
                for (int m = 0; m < M; ++m) {
                    const double xv = voxels[i * M + m];
                    s1[m * Vn + nj] += pj * xv;
                    s2[m * Vn + nj] += pj * xv * xv;
                }
            } else {
                outside[0] += pj;
                for (int m = 0; m < M; ++m) {
                    const double xv = voxels[i * M + m];
                    outside[1 + m] += pj * xv;
                    outside[1 + M + m] += pj * xv * xv;
                }
            }
            for (int q = 0; q < N; ++q) acc[q] += pj * (double)node[j][q];
        }
        for (int q = 0; q < N; ++q) dream[i * N + q] = acc[q];
    }
    return mll;
}

/* solve_linear_system (:348-389): Gaussian elimination with partial pivoting on [A | b] */
static void ssdf_solve(int n, const double *A, const double *b, double *x) {
    double aug[8][9];
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) aug[i][j] = A[i * n + j];
        aug[i][n] = b[i];
    }
    for (int i = 0; i < n; ++i) {
        int piv = i;
        for (int j = i + 1; j < n; ++j)
            if (fabs(aug[j][i]) > fabs(aug[piv][i])) piv = j;
        if (piv != i)
            for (int k = 0; k <= n; ++k) {
                const double t = aug[i][k];
                aug[i][k] = aug[piv][k];
                aug[piv][k] = t;
            }
        for (int j = i + 1; j < n; ++j) {
            const double f = aug[j][i] / aug[i][i];
            for (int k = i; k <= n; ++k) aug[j][k] -= f * aug[i][k];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = 0.0;
        for (int j = i + 1; j < n; ++j) s += aug[i][j] * x[j];
        x[i] = (aug[i][n] - s) / aug[i][i];
    }
}

/* update_parameters (:200-203): update_coefficients (:205-290, EM branch) then update_sigma
 * (:292-346), from the accumulators of orc_ssdf_estep; then compute_cost (:72-89).  With
 * update == 0 only the cost. */
/* sample_parameters (:459-463): update_coefficients and update_sigma with sample = true.
 * Coefficients (reg_across_features 0): x = solve(A, b_m), then sample_multivariate_normal(x, A)
 * as written (:392-427): L = chol(A) and coefficient i = x_i + sum_{j<=i} L_ij z_ij, a fresh
 * standard normal per term (Philox ctr {(m * 8 + i) * 8 + j, sweep, 8, chain}, Box-Muller on
 * words 0 and 1).  sigma_m = 1 / g, g ~ Gamma(shape den / 2, scale 2 / num_m)
 * (sample_inverse_gamma(den / 2, num_m / 2), :429-432; tag 9, index m), num_m with the drawn
 * coefficients.  Returns 1 when a gamma draw hit its attempt cap. */
int orc_ssdf_sample(orc_ssdf *p, const double *nodes, int nxn, int nyn, int nzn,
                    const double *gamma, const double *s1, const double *s2,
                    const double *outside, uint64_t seed, uint32_t sweep, uint32_t chain) {
    const int M = p->M, F = p->F;
    const long Vn = (long)nxn * nyn * nzn;
    double eff = outside[0];
    for (long j = 0; j < Vn; ++j) eff += gamma[j];
    if (!p->rfa) {
        double A[64] = {0}, b[64] = {0}, x[8], Lc[64] = {0};
        for (long j = 0; j < Vn; ++j)
            for (int f1 = 0; f1 < F; ++f1)
                for (int f2 = 0; f2 < F; ++f2)
                    A[f1 * F + f2] += nodes[j * F + f1] * nodes[j * F + f2] * gamma[j];
        for (int m = 0; m < M; ++m)
            for (long j = 0; j < Vn; ++j)
                for (int f = 0; f < F; ++f) b[m * F + f] += s1[m * Vn + j] * nodes[j * F + f];
        for (int i = 0; i < F; ++i)
            for (int j = 0; j <= i; ++j) {
                double sum = 0.0;
                for (int k = 0; k < j; ++k) sum += Lc[i * F + k] * Lc[j * F + k];
                Lc[i * F + j] = i == j ? sqrt(A[j * F + j] - sum) : (A[i * F + j] - sum) / Lc[j * F + j];
            }
        for (int m = 0; m < M; ++m) {
            ssdf_solve(F, A, b + m * F, x);
            for (int i = 0; i < F; ++i) {
                double v = x[i];
                for (int j = 0; j <= i; ++j) {
                    uint32_t r[4];
                    philox_draw(seed, (uint32_t)((m * 8 + i) * 8 + j), sweep, 8u, chain, r);
                    v += Lc[i * F + j] * sqrt(-2.0 * log(u01_d32(r[0]))) *
                         cos(2.0 * PI_D * u01_d32(r[1]));
                }
                p->coeff[m * F + i] = v;
            }
        }
    }
    int capped = 0;
    for (int m = 0; m < M; ++m) {
        double num = 0.0;
        for (long j = 0; j < Vn; ++j) {
            const double t = ssdf_pred(p, nodes, j, m);
            num += s2[m * Vn + j] + (-2.0 * s1[m * Vn + j] * t) + gamma[j] * t * t;
        }
        num += outside[1 + M + m];
        num += 2.0 * p->alpha0 * p->beta0;
        const double den = eff + 2.0 * p->alpha0;
        const double g = orc_gamma_sample(0.5 * den, seed, (uint32_t)m, sweep, 9u, chain, &capped) *
                         (2.0 / num);
        p->sigma[m] = 1.0 / g;
    }
    return capped;
}

double orc_ssdf_update(orc_ssdf *p, const double *nodes, int nxn, int nyn, int nzn,
                       const double *gamma, const double *s1, const double *s2,
                       const double *outside, int update) {
    const int M = p->M, F = p->F;
    const long Vn = (long)nxn * nyn * nzn;
    if (update) {
        double eff = outside[0];
        for (long j = 0; j < Vn; ++j) eff += gamma[j];
        if (!p->rfa) {
            double A[64] = {0}, b[64] = {0}, x[8];
            for (long j = 0; j < Vn; ++j)
                for (int f1 = 0; f1 < F; ++f1)
                    for (int f2 = 0; f2 < F; ++f2)
                        A[f1 * F + f2] += nodes[j * F + f1] * nodes[j * F + f2] * gamma[j];
            for (int m = 0; m < M; ++m)
                for (long j = 0; j < Vn; ++j)
                    for (int f = 0; f < F; ++f) b[m * F + f] += s1[m * Vn + j] * nodes[j * F + f];
            for (int m = 0; m < M; ++m) {
                ssdf_solve(F, A, b + m * F, x);
                for (int f = 0; f < F; ++f) p->coeff[m * F + f] = x[f];
            }
        }
        for (int m = 0; m < M; ++m) {
            double num = 0.0;
            for (long j = 0; j < Vn; ++j) {
                const double t = ssdf_pred(p, nodes, j, m);
                num += s2[m * Vn + j] + (-2.0 * s1[m * Vn + j] * t) + gamma[j] * t * t;
            }
            num += outside[1 + M + m];
            num += 2.0 * p->alpha0 * p->beta0;
            p->sigma[m] = num / (eff + 2.0 * p->alpha0);
        }
    }
    const double a = p->alpha0, bb = p->alpha0 * p->beta0;
    double cost = 0.0;
    for (int m = 0; m < M; ++m) {
        const double x = p->sigma[m];
        cost += -(a * log(bb) - lgamma(a) + (-a - 1.0) * log(x) - bb / x);
    }
    return cost;
}

