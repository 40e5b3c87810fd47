// Direct-evaluation implementation of the FFTW3 subset declared in fftw3.h (test infrastructure).
#include "fftw3.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {
constexpr double kPi = 3.14159265358979323846;

struct Plan {
    int rank = 0;
    int n[3] = {1, 1, 1};
    bool complex = false;
    int sign = -1;
    fftw_r2r_kind kind[3] = {FFTW_REDFT10, FFTW_REDFT10, FFTW_REDFT10};
    double *rin = nullptr, *rout = nullptr;
    fftw_complex *cin = nullptr, *cout = nullptr;
};

// one r2r transform along an axis of length n, stride s, for every line
void r2r_axis(double *a, int n, long outer, long s, fftw_r2r_kind kind) {
    std::vector<double> line(n), res(n);
    for (long o = 0; o < outer * s; ++o) {
        const long b = (o / s) * (long)n * s + (o % s);
        for (int j = 0; j < n; ++j) line[j] = a[b + (long)j * s];
        for (int k = 0; k < n; ++k) {
            double acc = 0.0;
            if (kind == FFTW_REDFT10) {
                for (int j = 0; j < n; ++j) {
                    const long m = ((long)(2 * j + 1) * k) % (4L * n);
                    acc += line[j] * std::cos(kPi * (double)m / (2.0 * n));
                }
                acc *= 2.0;
            } else {  // FFTW_REDFT01
                acc = line[0];
                for (int j = 1; j < n; ++j) {
                    const long m = ((long)j * (2 * k + 1)) % (4L * n);
                    acc += 2.0 * line[j] * std::cos(kPi * (double)m / (2.0 * n));
                }
            }
            res[k] = acc;
        }
        for (int k = 0; k < n; ++k) a[b + (long)k * s] = res[k];
    }
}

void dft_axis(fftw_complex *a, int n, long outer, long s, int sign) {
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
void fftw_plan_with_nthreads(int) {}
int fftw_export_wisdom_to_filename(const char *) { return 1; }
int fftw_import_wisdom_from_filename(const char *) { return 0; }

}  // extern "C"
