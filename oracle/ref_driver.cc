/* ref_driver.cc -- extern "C" entry points into the UNMODIFIED reference code.
 *
 * TEST INFRASTRUCTURE ONLY. Compiled by oracle/Makefile together with the
 * reference sources where they lie (never copied) into oracle/_ref/
 * libconan_ref.so. It instantiates the reference's own templates and classes
 * (md_cic, gradient_2nd_order, LinearInterpolation<Gradient>, Zeldovich,
 * Gravity, LeapFrog, generate_random_field, compute_potential) so tests can
 * pin the CPU restatement in conan_oracle.cc against them, and bench.py can
 * time the reference's own PM step as the CPU baseline.
 */
#include "../base/system.hh"
#include "../base/format.hh"
#include "../ic/ic.hh"
#include "cosmology.hh"
#include "leapfrog.hh"
#include "nbody.hh"

#include <chrono>
#include <cstdio>
#include <fcntl.h>
#include <omp.h>
#include <unistd.h>

using namespace System;
using namespace Conan;

namespace {

/* The reference prints progress dots on stdout from Gravity::kick; keep the
 * caller's stdout clean (bench.py prints one JSON line there). */
struct QuietStdout {
    int saved;
    QuietStdout() {
        std::cout.flush();
        fflush(stdout);
        saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        dup2(dn, 1);
        close(dn);
    }
    ~QuietStdout() {
        std::cout.flush();
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

Header ic_header(int dim, int mbits, double L, double ns, int smooth, int scale_free,
                 double scale, double sigma, unsigned seed) {
    Header H;
    H["dim"] = Misc::format(dim);
    H["mbits"] = Misc::format(mbits);
    H["size"] = Misc::format(L);
    H["ns"] = Misc::format(ns);
    H["smooth"] = smooth ? "1" : "0";
    H["scale-free"] = scale_free ? "1" : "0";
    H["scale"] = Misc::format(scale);
    H["sigma"] = Misc::format(sigma);
    H["seed"] = Misc::format(seed);
    H["Omega0"] = "0.32";
    H["H0"] = "69.0";
    H["N"] = Misc::format(1 << mbits);
    return H;
}

template <unsigned R>
void md_cic_t(int N, double L, const double *X, size_t n, double m, double *out) {
    auto box = BoxMaker(N, L).box<R>();
    Array<double> res(box->size());
    Array<dVector<R>> P(n);
    for (size_t i = 0; i < n; ++i)
        for (unsigned k = 0; k < R; ++k) P[i][k] = X[i * R + k];
    md_cic<R>(box, res, P, m);
    for (size_t i = 0; i < box->size(); ++i) out[i] = res[i];
}

template <unsigned R>
void interp_t(int N, double L, const double *phi, const double *X, size_t n, double *out) {
    auto box = BoxMaker(N, L).box<R>();
    Array<double> f(box->size());
    for (size_t i = 0; i < box->size(); ++i) f[i] = phi[i];
    Gradient<R> g(box, f);
    LinearInterpolation<Gradient<R>, R> A(box, g);
    for (size_t i = 0; i < n; ++i) {
        dVector<R> x;
        for (unsigned k = 0; k < R; ++k) x[k] = X[i * R + k];
        dVector<R> v = A(x);
        for (unsigned k = 0; k < R; ++k) out[i * R + k] = v[k];
    }
}

template <unsigned R>
void zeldovich_t(int N, double L, const double *phi, double a_pos, double a_mom, double *X,
                 double *P) {
    auto box = BoxMaker(N, L).box<R>();
    Array<double> f(box->size());
    for (size_t i = 0; i < box->size(); ++i) f[i] = phi[i];
    Zeldovich<R> ZA(box, f);
    Array<dVector<R>> x(box->size()), p(box->size());
    ZA.x(x, a_pos);
    ZA.p(p, a_mom);
    for (size_t i = 0; i < box->size(); ++i)
        for (unsigned k = 0; k < R; ++k) {
            X[i * R + k] = x[i][k];
            P[i * R + k] = p[i][k];
        }
}

template <unsigned R>
double time_steps_t(int Nm, int f, double L, double H0, double Om, double OL, const double *phi,
                    double a0, double da, unsigned n, double *t_init) {
    auto mbox = BoxMaker(Nm, L).box<R>();
    auto fbox = BoxMaker(f * Nm, L).box<R>();
    Array<double> p(mbox->size());
    for (size_t i = 0; i < mbox->size(); ++i) p[i] = phi[i];
    Cosmology cosmos(H0, Om, OL);
    QuietStdout quiet;
    auto t0 = std::chrono::steady_clock::now();
    Gravity<R> G("bench", mbox, fbox, p, cosmos, false, FMT_CONAN);
    G.init(a0, a0 + da / 2);
    auto t1 = std::chrono::steady_clock::now();
    double a = a0;
    for (unsigned i = 0; i < n; ++i) {
        G.drift(a, da);
        G.kick(a + da / 2, da);
        a += da;
    }
    auto t2 = std::chrono::steady_clock::now();
    if (t_init) *t_init = std::chrono::duration<double>(t1 - t0).count();
    return std::chrono::duration<double>(t2 - t1).count();
}

/* One solver state, one leapfrog step per entry of threads[]: step i runs
 * with omp_set_num_threads(threads[i]) and its seconds go to seconds[i]. */
template <unsigned R>
double time_threads_t(int Nm, int f, double L, double H0, double Om, double OL, const double *phi,
                      double a0, double da, int nt, const int *threads, double *seconds) {
    auto mbox = BoxMaker(Nm, L).box<R>();
    auto fbox = BoxMaker(f * Nm, L).box<R>();
    Array<double> p(mbox->size());
    for (size_t i = 0; i < mbox->size(); ++i) p[i] = phi[i];
    Cosmology cosmos(H0, Om, OL);
    QuietStdout quiet;
    const int saved = omp_get_max_threads();
    auto t0 = std::chrono::steady_clock::now();
    Gravity<R> G("bench", mbox, fbox, p, cosmos, false, FMT_CONAN);
    G.init(a0, a0 + da / 2);
    auto t1 = std::chrono::steady_clock::now();
    double a = a0;
    for (int i = 0; i < nt; ++i) {
        omp_set_num_threads(threads[i] > 0 ? threads[i] : saved);
        auto s0 = std::chrono::steady_clock::now();
        G.drift(a, da);
        G.kick(a + da / 2, da);
        auto s1 = std::chrono::steady_clock::now();
        seconds[i] = std::chrono::duration<double>(s1 - s0).count();
        a += da;
    }
    omp_set_num_threads(saved);
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // namespace

extern "C" {

int ref_max_threads(void) { return omp_get_max_threads(); }

/* Conan::generate_random_field (src/ic/ic.cc:148-161) on a header built from
 * the given `ic` options. */
void ref_generate_random_field(int dim, int mbits, double L, double ns, int smooth,
                               int scale_free, double scale, double sigma, unsigned seed,
                               double *out) {
    Header H = ic_header(dim, mbits, L, ns, smooth, scale_free, scale, sigma, seed);
    Array<double> D = Conan::generate_random_field(H);
    for (size_t i = 0; i < D.size(); ++i) out[i] = D[i];
}

/* Conan::compute_potential (src/ic/ic.cc:163-176), in place. */
void ref_compute_potential(int dim, int mbits, double L, double *data) {
    Header H = ic_header(dim, mbits, L, 0, 0, 1, 8, 0.83, 0);
    size_t n = 1;
    for (int i = 0; i < dim; ++i) n *= (size_t)1 << mbits;
    Array<double> D(n);
    for (size_t i = 0; i < n; ++i) D[i] = data[i];
    Conan::compute_potential(H, D);
    for (size_t i = 0; i < n; ++i) data[i] = D[i];
}

/* md_cic<R> (src/run/numeric.hh:106-139). */
void ref_md_cic(int dim, int N, double L, const double *X, size_t n, double m, double *out) {
    switch (dim) {
        case 1: md_cic_t<1>(N, L, X, n, m, out); break;
        case 2: md_cic_t<2>(N, L, X, n, m, out); break;
        case 3: md_cic_t<3>(N, L, X, n, m, out); break;
    }
}

/* LinearInterpolation<Gradient<R>,R> (src/run/numeric.hh:6-45,72-103). */
void ref_interp_gradient(int dim, int N, double L, const double *phi, const double *X, size_t n,
                         double *out) {
    switch (dim) {
        case 1: interp_t<1>(N, L, phi, X, n, out); break;
        case 2: interp_t<2>(N, L, phi, X, n, out); break;
        case 3: interp_t<3>(N, L, phi, X, n, out); break;
    }
}

/* Zeldovich<R>::x / ::p (src/run/nbody.hh:26-51). */
void ref_zeldovich(int dim, int N, double L, const double *phi, double a_pos, double a_mom,
                   double *X, double *P) {
    switch (dim) {
        case 1: zeldovich_t<1>(N, L, phi, a_pos, a_mom, X, P); break;
        case 2: zeldovich_t<2>(N, L, phi, a_pos, a_mom, X, P); break;
        case 3: zeldovich_t<3>(N, L, phi, a_pos, a_mom, X, P); break;
    }
}

/* Times n leapfrog steps of the reference's Gravity<R> solver
 * (src/run/nbody.hh:53-133) after its init; returns the seconds spent in
 * the steps and stores the init time in *t_init. */
double ref_time_steps(int dim, int Nm, int f, double L, double H0, double Om, double OL,
                      const double *phi, double a0, double da, unsigned n, double *t_init) {
    switch (dim) {
        case 1: return time_steps_t<1>(Nm, f, L, H0, Om, OL, phi, a0, da, n, t_init);
        case 2: return time_steps_t<2>(Nm, f, L, H0, Om, OL, phi, a0, da, n, t_init);
        case 3: return time_steps_t<3>(Nm, f, L, H0, Om, OL, phi, a0, da, n, t_init);
    }
    return -1;
}

/* Times one leapfrog step of the reference's Gravity<R> (src/run/nbody.hh:
 * 97-133) per entry of threads[] (0: all threads) on one solver state, after
 * one init; returns the init seconds, the steps' seconds in seconds[]. */
double ref_time_threads(int dim, int Nm, int f, double L, double H0, double Om, double OL, const double *phi,
                        double a0, double da, int nt, const int *threads, double *seconds) {
    switch (dim) {
        case 1: return time_threads_t<1>(Nm, f, L, H0, Om, OL, phi, a0, da, nt, threads, seconds);
        case 2: return time_threads_t<2>(Nm, f, L, H0, Om, OL, phi, a0, da, nt, threads, seconds);
        case 3: return time_threads_t<3>(Nm, f, L, H0, Om, OL, phi, a0, da, nt, threads, seconds);
    }
    return -1;
}

}  // extern "C"
