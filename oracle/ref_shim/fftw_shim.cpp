// Implementation of the FFTW3 subset declared in fftw3.h (test infrastructure): the real-to-real
// DCTs in O(n log n) (Makhoul, "A fast cosine transform in one and multiple dimensions", IEEE
// Trans. ASSP 28, 1980: a length-n complex FFT and a twiddle per output; mixed-radix Cooley-Tukey
// FFT), lines threaded with OpenMP at the plan's thread count; the complex DFTs by direct
// evaluation on lines of up to kDirectMax points (the sizes of the golden fixtures, whose order of
// operations the FP64 oracle restates) and by the same mixed-radix FFT on longer lines, threaded
// over lines.  FFTW's unnormalised conventions throughout.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {
constexpr double kPi = 3.14159265358979323846;
int g_threads = 1;
typedef std::complex<double> cd;

// out[k] = sum_j in[j * stride] e^{sign 2 pi i jk / n}, n a divisor of N = the length of the
// table e^{-2 pi i t / N} (recursive decimation in time by the smallest prime factor; scratch
// holds 2n values)
void fft_rec(const cd *in, long stride, cd *out, int n, int sign, const cd *table, int N,
             cd *scratch) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    int p = 2;
    while (n % p) ++p;
    const int m = n / p;
    const int step = N / n;  // e^{-2 pi i t / n} = table[t * step]
    // sub-transforms of the p decimated sequences, stored at scratch[r * m .. r * m + m)
    for (int r = 0; r < p; ++r)
        fft_rec(in + (long)r * stride, stride * p, scratch + (long)r * m, m, sign, table, N,
                scratch + n);
    for (int k = 0; k < m; ++k)
        for (int q = 0; q < p; ++q) {
            const int kk = k + q * m;
            cd acc = scratch[k];
            for (int r = 1; r < p; ++r) {
                const cd t = table[(long)(((long)r * kk) % n) * step];
                acc += scratch[(long)r * m + k] * (sign < 0 ? t : std::conj(t));
            }
            out[kk] = acc;
        }
}

// per-length tables of one thread: the DCT twiddles e^{-i pi k / (2n)} and the FFT scratch
struct DctWork {
    int n = 0;
    std::vector<cd> tw, table, v, V, scratch;
    void init(int len) {
        if (n == len) return;
        n = len;
        tw.resize(n);
        table.resize(n);
        for (int k = 0; k < n; ++k) {
            tw[k] = cd(std::cos(kPi * k / (2.0 * n)), -std::sin(kPi * k / (2.0 * n)));
            table[k] = cd(std::cos(2.0 * kPi * k / n), -std::sin(2.0 * kPi * k / n));
        }
        v.resize(n);
        V.resize(n);
        scratch.resize((size_t)4 * n + 8);
    }
};

// REDFT10: y_k = 2 sum_j x_j cos(pi (2j + 1) k / (2n)) = 2 Re(e^{-i pi k/(2n)} V_k), V the DFT of
// the even samples followed by the odd ones reversed
void redft10(const double *x, double *y, DctWork &w) {
    const int n = w.n;
    for (int j = 0; 2 * j < n; ++j) w.v[j] = x[2 * j];
    for (int j = 0; 2 * j + 1 < n; ++j) w.v[n - 1 - j] = x[2 * j + 1];
    fft_rec(w.v.data(), 1, w.V.data(), n, -1, w.table.data(), n, w.scratch.data());
    for (int k = 0; k < n; ++k) y[k] = 2.0 * (w.tw[k] * w.V[k]).real();
}

// REDFT01 (= 2n times the inverse of REDFT10): V_k = e^{i pi k/(2n)} (x_k - i x_{n-k}) / 2
// (x_n = 0), w = the unnormalised inverse DFT of V, y_{2j} = 2 Re w_j, y_{2j+1} = 2 Re w_{n-1-j}
void redft01(const double *x, double *y, DctWork &w) {
    const int n = w.n;
    for (int k = 0; k < n; ++k) {
        const double xr = x[k], xi = k ? -x[n - k] : 0.0;
        w.v[k] = std::conj(w.tw[k]) * cd(xr, xi) * 0.5;
    }
    fft_rec(w.v.data(), 1, w.V.data(), n, +1, w.table.data(), n, w.scratch.data());
    for (int j = 0; 2 * j < n; ++j) y[2 * j] = 2.0 * w.V[j].real();
    for (int j = 0; 2 * j + 1 < n; ++j) y[2 * j + 1] = 2.0 * w.V[n - 1 - j].real();
}

struct Plan {
    int rank = 0;
    int n[3] = {1, 1, 1};
    bool complex = false;
    int sign = -1;
    fftw_r2r_kind kind[3] = {FFTW_REDFT10, FFTW_REDFT10, FFTW_REDFT10};
    double *rin = nullptr, *rout = nullptr;
    fftw_complex *cin = nullptr, *cout = nullptr;
};

// one r2r transform along an axis of length n, stride s, for every line (lines in parallel)
void r2r_axis(double *a, int n, long outer, long s, fftw_r2r_kind kind) {
    const long lines = outer * s;
#pragma omp parallel num_threads(g_threads)
    {
        DctWork w;
        w.init(n);
        std::vector<double> line(n), res(n);
#pragma omp for schedule(static)
        for (long o = 0; o < lines; ++o) {
            const long b = (o / s) * (long)n * s + (o % s);
            for (int j = 0; j < n; ++j) line[j] = a[b + (long)j * s];
            if (kind == FFTW_REDFT10) redft10(line.data(), res.data(), w);
            else redft01(line.data(), res.data(), w);
            for (int k = 0; k < n; ++k) a[b + (long)k * s] = res[k];
        }
    }
}

constexpr int kDirectMax = 32;

void dft_axis_fft(fftw_complex *a, int n, long outer, long s, int sign) {
    const long lines = outer * s;
#pragma omp parallel num_threads(g_threads)
    {
        std::vector<cd> table(n), line(n), res(n), scratch((size_t)4 * n + 8);
        for (int k = 0; k < n; ++k)
            table[k] = cd(std::cos(2.0 * kPi * k / n), -std::sin(2.0 * kPi * k / n));
#pragma omp for schedule(static)
        for (long o = 0; o < lines; ++o) {
            const long b = (o / s) * (long)n * s + (o % s);
            for (int j = 0; j < n; ++j)
                line[j] = cd(a[b + (long)j * s][0], a[b + (long)j * s][1]);
            fft_rec(line.data(), 1, res.data(), n, sign, table.data(), n, scratch.data());
            for (int k = 0; k < n; ++k) {
                a[b + (long)k * s][0] = res[k].real();
                a[b + (long)k * s][1] = res[k].imag();
            }
        }
    }
}

void dft_axis(fftw_complex *a, int n, long outer, long s, int sign) {
    if (n > kDirectMax) {
        dft_axis_fft(a, n, outer, s, sign);
        return;
    }
    std::vector<double> re(n), im(n), cr(n), ci(n);
    for (long o = 0; o < outer * s; ++o) {
        const long b = (o / s) * (long)n * s + (o % s);
        for (int j = 0; j < n; ++j) { re[j] = a[b + (long)j * s][0]; im[j] = a[b + (long)j * s][1]; }
        for (int k = 0; k < n; ++k) {
            double ar = 0.0, ai = 0.0;
            for (int j = 0; j < n; ++j) {
                const long m = ((long)j * k) % n;
                const double c = std::cos(2.0 * kPi * (double)m / n);
                const double sn = sign * std::sin(2.0 * kPi * (double)m / n);
                ar += re[j] * c - im[j] * sn;
                ai += re[j] * sn + im[j] * c;
            }
            cr[k] = ar; ci[k] = ai;
        }
        for (int k = 0; k < n; ++k) { a[b + (long)k * s][0] = cr[k]; a[b + (long)k * s][1] = ci[k]; }
    }
}
}  // namespace

struct binder_shim_plan : Plan {};

extern "C" {

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out, fftw_r2r_kind k0,
                           fftw_r2r_kind k1, unsigned) {
    auto *p = new binder_shim_plan();
    p->rank = 2; p->n[0] = n0; p->n[1] = n1; p->kind[0] = k0; p->kind[1] = k1;
    p->rin = in; p->rout = out;
    return p;
}

fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double *in, double *out, fftw_r2r_kind k0,
                           fftw_r2r_kind k1, fftw_r2r_kind k2, unsigned) {
    auto *p = new binder_shim_plan();
    p->rank = 3; p->n[0] = n0; p->n[1] = n1; p->n[2] = n2;
    p->kind[0] = k0; p->kind[1] = k1; p->kind[2] = k2;
    p->rin = in; p->rout = out;
    return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
    auto *p = new binder_shim_plan();
    p->rank = 2; p->n[0] = n0; p->n[1] = n1; p->complex = true; p->sign = sign;
    p->cin = in; p->cout = out;
    return p;
}

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned) {
    auto *p = new binder_shim_plan();
    p->rank = 3; p->n[0] = n0; p->n[1] = n1; p->n[2] = n2; p->complex = true; p->sign = sign;
    p->cin = in; p->cout = out;
    return p;
}

void fftw_execute(const fftw_plan p) {
    long total = 1;
    for (int d = 0; d < p->rank; ++d) total *= p->n[d];
    // axis d: length n[d], stride = product of later dims, outer = product of earlier dims
    if (p->complex) {
        if (p->cout != p->cin) std::memcpy(p->cout, p->cin, sizeof(fftw_complex) * total);
        for (int d = p->rank - 1; d >= 0; --d) {
            long s = 1, outer = 1;
            for (int e = d + 1; e < p->rank; ++e) s *= p->n[e];
            for (int e = 0; e < d; ++e) outer *= p->n[e];
            dft_axis(p->cout, p->n[d], outer, s, p->sign);
        }
    } else {
        if (p->rout != p->rin) std::memcpy(p->rout, p->rin, sizeof(double) * total);
        for (int d = p->rank - 1; d >= 0; --d) {
            long s = 1, outer = 1;
            for (int e = d + 1; e < p->rank; ++e) s *= p->n[e];
            for (int e = 0; e < d; ++e) outer *= p->n[e];
            r2r_axis(p->rout, p->n[d], outer, s, p->kind[d]);
        }
    }
}

void fftw_destroy_plan(fftw_plan p) { delete p; }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { g_threads = n > 0 ? n : 1; }
int fftw_export_wisdom_to_filename(const char *) { return 1; }
int fftw_import_wisdom_from_filename(const char *) { return 0; }

}  // extern "C"
