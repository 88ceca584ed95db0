/* conan_oracle.cc -- FP64 CPU restatement of conan's PM path and initial conditions.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA
 * product: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it, and the product never calls it. Every function restates the
 * reference algorithm it cites (paths relative to the reference project root)
 * in the same operation order, in double precision, so that its results match
 * the reference's own CPU run to rounding. Loops whose iterations each write
 * only their own element (per particle or per cell) run on OpenMP threads, so
 * the results do not depend on the thread count; every sum over particles or
 * cells (the deposits, variances, dot products) runs serially in index order. It is pinned
 * against golden outputs written by the unmodified reference binary
 * (tests/golden/make_golden.py).
 *
 * Layout conventions are the reference's: meshes are N^R doubles with axis 0
 * fastest (src/base/box.hh:51-53); particle vectors are arrays of R doubles
 * per particle (mVector<double,R>, src/base/mvector.hh:16-19).
 */
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "fftw_shim/fftw3.h"

typedef std::complex<double> cplx;

namespace {

size_t ipow(size_t n, int r) {
    size_t s = 1;
    for (int i = 0; i < r; ++i) s *= n;
    return s;
}

/* Integer modulus with the mathematical sign, src/base/misc.hh:135-139. */
inline int imod(int a, int b) { return a < 0 ? b + (a % b) : a % b; }

/* Floating modulus with truncating casts, src/base/misc.hh:144-148. */
inline double dmod(double a, double b) {
    if (a < 0) return a - static_cast<int>(a / b - 1) * b;
    return a - static_cast<int>(a / b) * b;
}

/* Linear index of an R-vector with periodic wrap, axis 0 fastest:
 * Box::idx, src/base/box.hh:75-81. */
inline size_t box_idx(const int *x, int R, int N) {
    size_t a = 0, s = 1;
    for (int i = 0; i < R; ++i) {
        a += (size_t)imod(x[i], N) * s;
        s *= (size_t)N;
    }
    return a;
}

/* Decode a linear index into an R-vector, MdRange::operator[],
 * src/base/mdrange.hh:106-115. */
inline void decode(size_t idx, int R, int N, int *out) {
    for (int i = 0; i < R; ++i) {
        out[i] = (int)(idx % (size_t)N);
        idx = (idx - out[i]) / (size_t)N;
    }
}

/* Signed wave number of index i, Fourier::kspace, src/base/fourier.hh:42-55. */
inline double wave(int i, int N, double L) {
    long a = i;
    return ((unsigned)i > (unsigned)N / 2 ? a - (long)N : a) * (2 * M_PI / L);
}

/* Complex DFT over an R-cube of side N, unnormalised (src/base/fft.cc:15-38). */
void dft(std::vector<cplx> &in, std::vector<cplx> &out, int R, int N, int sign) {
    std::vector<int> shape(R, N);
    fftw_plan p = fftw_plan_dft(R, shape.data(), reinterpret_cast<fftw_complex *>(in.data()),
                                reinterpret_cast<fftw_complex *>(out.data()), sign, FFTW_ESTIMATE);
    fftw_execute(p);
    fftw_destroy_plan(p);
}

void kvec(size_t idx, int R, int N, double L, double *k) {
    int x[8];
    decode(idx, R, N, x);
    for (int i = 0; i < R; ++i) k[i] = wave(x[i], N, L);
}

double sqr(const double *k, int R) {
    double v = 0;
    for (int i = 0; i < R; ++i) v += k[i] * k[i];
    return v;
}

/* Fourier::scale(t), src/base/fourier.hh:79-91. */
double scale_filter(const double *k, int R, double t) {
    double v = 1.0;
    for (int i = 0; i < R; ++i) v *= std::exp(t * (std::cos(k[i]) - 1));
    return v;
}

}  // namespace

extern "C" {

/* Seeded unit white noise in memory order: Gaussian_white_noise(seed)
 * (src/base/misc.hh:179-188) filled by generate() (src/ic/ic.cc:55-56).
 * The sequence is defined by libstdc++'s std::mt19937 and
 * std::normal_distribution<double>, called here as library routines. */
void oracle_noise_mt19937(unsigned long seed, size_t n, double *out) {
    std::mt19937 rng(seed);
    std::normal_distribution<double> normal;
    for (size_t i = 0; i < n; ++i) out[i] = normal(rng);
}

/* Unnormalised complex DFT of an R-cube (for tests of the shim FFT). */
void oracle_dft(int R, int N, const double *in_ri, double *out_ri, int sign) {
    size_t n = ipow(N, R);
    std::vector<cplx> a(n), b(n);
    std::memcpy(a.data(), in_ri, n * sizeof(cplx));
    dft(a, b, R, N, sign);
    std::memcpy(out_ri, b.data(), n * sizeof(cplx));
}

/* Scale-free Gaussian random field, _generate_random_field<R> scale-free
 * branch, src/ic/ic.cc:37-83. `noise` holds N^R unit normals in memory
 * order; `dens` receives the normalised density. */
void oracle_grf_scale_free(int R, int mbits, double L, double slope, int smooth,
                           double scale, double sigma_norm, const double *noise,
                           double *dens) {
    int N = 1 << mbits;
    size_t size = ipow(N, R);
    std::vector<cplx> in(size), out(size);
    for (size_t i = 0; i < size; ++i) in[i] = noise[i];
    double t = scale * N / L; /* Fourier::scale<R>(sigma * N/L), ic.cc:63 */
    auto PS = [&](size_t idx, bool with_s) {
        double k[8];
        kvec(idx, R, N, (double)N, k); /* kspace<R>(N, N), ic.cc:64 */
        double p = std::sqrt(std::pow(std::sqrt(sqr(k, R)), slope));
        double s = with_s ? scale_filter(k, R, t) : 1.0;
        return cplx(p) * cplx(s);
    };
    dft(in, out, R, N, FFTW_FORWARD);
    for (size_t i = 0; i < size; ++i) in[i] = out[i] * PS(i, true);
    in[0] = 0;
    dft(in, out, R, N, FFTW_BACKWARD);
    for (size_t i = 0; i < size; ++i) in[i] = noise[i]; /* copy(dens, fft.in), ic.cc:70 */
    std::vector<double> d(size);
    for (size_t i = 0; i < size; ++i) d[i] = out[i].real() / (double)size;
    double acc = 0;
    for (size_t i = 0; i < size; ++i) acc += d[i] * d[i];
    double var = acc / (double)size;
    dft(in, out, R, N, FFTW_FORWARD);
    for (size_t i = 0; i < size; ++i) {
        if (smooth)
            in[i] = out[i] * PS(i, true);
        else
            in[i] = out[i] * PS(i, false);
    }
    in[0] = 0;
    dft(in, out, R, N, FFTW_BACKWARD);
    double s = (double)size * std::sqrt(var) / sigma_norm;
    for (size_t i = 0; i < size; ++i) dens[i] = out[i].real() / s;
}

/* CDM branch: filter sqrt(P(|k|)) with the BBKS-like transfer function of
 * CDM<R>, src/ic/ic.cc:14-35, applied at src/ic/ic.cc:84-97. */
void oracle_grf_cdm(int R, int mbits, double L, double Omega0, double H0, double ns,
                    const double *noise, double *dens) {
    int N = 1 << mbits;
    size_t size = ipow(N, R);
    double res = L / N;
    const double e = std::exp(1), Theta = 2.7255 / 2.7, h = H0 / 100.0, A = 1122670;
    std::vector<cplx> in(size), out(size);
    for (size_t i = 0; i < size; ++i) in[i] = noise[i];
    dft(in, out, R, N, FFTW_FORWARD);
    for (size_t i = 0; i < size; ++i) {
        double k[8];
        kvec(i, R, N, L, k);
        double kk = std::sqrt(sqr(k, R));
        double q = kk * std::pow(Theta, 2) / (Omega0 * h), L0 = std::log(2 * e + 1.8 * q),
               C0 = 14.2 + 731.0 / (1 + 62.5 * q), T0 = L0 / (L0 + C0 * std::pow(q, 2));
        double P = A * std::pow(kk, ns) * std::pow(T0, 2);
        in[i] = out[i] * cplx(std::sqrt(P));
    }
    in[0] = 0;
    dft(in, out, R, N, FFTW_BACKWARD);
    double s = (double)size * std::pow(res, 0.5 * R);
    for (size_t i = 0; i < size; ++i) dens[i] = out[i].real() / s;
}

/* Gravitational potential -1/k^2 in physical units, in place:
 * _compute_potential<R>, src/ic/ic.cc:100-117. */
void oracle_potential(int R, int mbits, double L, double *data) {
    int N = 1 << mbits;
    size_t size = ipow(N, R);
    std::vector<cplx> in(size), out(size);
    for (size_t i = 0; i < size; ++i) in[i] = data[i];
    dft(in, out, R, N, FFTW_FORWARD);
    for (size_t i = 0; i < size; ++i) {
        double k[8];
        kvec(i, R, N, L, k);
        in[i] = out[i] * cplx(-1. / sqr(k, R));
    }
    in[0] = 0;
    dft(in, out, R, N, FFTW_BACKWARD);
    for (size_t i = 0; i < size; ++i) data[i] = out[i].real() / (double)size;
}

/* Zel'dovich displacement record: _compute_displacement<R>,
 * src/ic/ic.cc:119-146. psi has R doubles per cell. */
void oracle_displacement(int R, int mbits, double L, const double *pot, double *psi) {
    int N = 1 << mbits;
    size_t size = ipow(N, R);
    std::vector<cplx> in(size), out(size), phif(size);
    for (size_t i = 0; i < size; ++i) in[i] = pot[i];
    dft(in, out, R, N, FFTW_FORWARD);
    phif = out;
    for (int c = 0; c < R; ++c) {
        for (size_t i = 0; i < size; ++i) {
            double k[8];
            kvec(i, R, N, (double)N, k);
            in[i] = phif[i] * (cplx(0, 1.0) * std::sin(k[c]));
        }
        dft(in, out, R, N, FFTW_BACKWARD);
        double s = (double)size / L * N;
        for (size_t i = 0; i < size; ++i) psi[i * R + c] = out[i].real() / s;
    }
}

/* 4-point finite-difference gradient of f at every node, divided by res:
 * gradient_2nd_order<R>, src/run/numeric.hh:48-70. */
void oracle_gradient(int R, int N, double L, const double *f, double *g) {
    size_t size = ipow(N, R);
    double res = L / N;
#pragma omp parallel for schedule(static)
    for (size_t x = 0; x < size; ++x) {
        int p0[8], q[8];
        decode(x, R, N, p0);
        for (int k = 0; k < R; ++k) {
            size_t id[4];
            int off[4] = {-2, -1, 1, 2};
            for (int j = 0; j < 4; ++j) {
                std::memcpy(q, p0, sizeof(int) * R);
                q[k] += off[j];
                id[j] = box_idx(q, R, N);
            }
            double v = f[id[0]] / 12. - 2 * f[id[1]] / 3. + 2 * f[id[2]] / 3. - f[id[3]] / 12.;
            g[x * R + k] = v / res;
        }
    }
}

/* Zel'dovich initial positions and momenta: Gravity::init,
 * src/run/nbody.hh:88-95, with Zeldovich<R>, src/run/nbody.hh:26-51.
 * X = q - a_pos u, P = -a_mom u, u = gradient of phi on the mass mesh. */
void oracle_zeldovich(int R, int Nm, double L, const double *phi, double a_pos, double a_mom,
                      double *X, double *P) {
    size_t size = ipow(Nm, R);
    std::vector<double> u(size * R);
    oracle_gradient(R, Nm, L, phi, u.data());
    double cell = L / Nm; /* grid_space: x[i] * (L/N), src/base/box.hh:11-24 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < size; ++i) {
        int q[8];
        decode(i, R, Nm, q);
        for (int k = 0; k < R; ++k) {
            X[i * R + k] = q[k] * cell - u[i * R + k] * a_pos;
            P[i * R + k] = u[i * R + k] * -a_mom;
        }
    }
}

/* Cloud-in-cell mass deposit: md_cic<R>, src/run/numeric.hh:106-139.
 * Summed serially in particle order (the reference's `omp critical` makes
 * its order thread-dependent; the sum is the same to rounding). */
void oracle_md_cic(int R, int N, double L, const double *X, size_t n, double m, double *out) {
    size_t size = ipow(N, R);
    double res = L / N;
    for (size_t i = 0; i < size; ++i) out[i] = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double p0[8], A[2][8];
        int origin[8];
        for (int k = 0; k < R; ++k) {
            p0[k] = dmod(X[i * R + k], L) / res;
            origin[k] = (int)p0[k];
            A[1][k] = p0[k] - origin[k];
            A[0][k] = 1 - A[1][k];
        }
        for (int j = 0; j < (1 << R); ++j) {
            double z = m;
            int c[8];
            for (int k = 0; k < R; ++k) {
                int b = (j >> k) & 1;
                z *= A[b][k];
                c[k] = origin[k] + b;
            }
            out[box_idx(c, R, N)] += z;
        }
    }
}

/* The `cic` tool's density, cic_run<R> (src/cic/cic.hh:49-81): X holds the
 * N^R absolute positions of a snapshot (AoS); out receives the Nf^R mesh,
 * Nf = f N. s = 1: md_cic with unit mass. s > 1: the displacement X - G is
 * interpolated linearly (LinearInterpolation, src/run/numeric.hh:6-45, on the
 * mass grid) at the points of an (N s)^R grid (grid_space, src/base/box.hh:
 * 11-24) and those points are deposited with mass (s N / Nf)^-R. */
void oracle_cic(int R, int N, double L, int f, int s, const double *X, double *out) {
    const int Nf = N * f;
    const size_t np = ipow(N, R);
    if (s == 1) {
        oracle_md_cic(R, Nf, L, X, np, 1.0, out);
        return;
    }
    const double res_m = L / N;
    std::vector<double> D(np * R);
    for (size_t i = 0; i < np; ++i) {
        size_t r = i;
        for (int k = 0; k < R; ++k) {
            D[i * R + k] = X[i * R + k] - (double)(r % N) * (L / N);
            r /= N;
        }
    }
    const int Ns = N * s;
    const size_t nsub = ipow(Ns, R);
    std::vector<double> Y(nsub * R);
    for (size_t j = 0; j < nsub; ++j) {
        double y[8], x[8], A[2][8];
        int origin[8];
        size_t r = j;
        for (int k = 0; k < R; ++k) {
            y[k] = (double)(r % Ns) * (L / Ns);
            r /= Ns;
            x[k] = y[k] / res_m;
            origin[k] = (int)x[k];
            A[1][k] = x[k] - origin[k];
            A[0][k] = 1 - A[1][k];
        }
        double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int b = 0; b < (1 << R); ++b) {
            double z = 1;
            int c[8];
            for (int k = 0; k < R; ++k) {
                int bk = (b >> k) & 1;
                z *= A[bk][k];
                c[k] = origin[k] + bk;
            }
            size_t id = box_idx(c, R, N);
            for (int k = 0; k < R; ++k) v[k] += D[id * R + k] * z;
        }
        for (int k = 0; k < R; ++k) Y[j * R + k] = y[k] + v[k];
    }
    const double a = std::pow(double(s * N) / double(Nf), -float(R));
    oracle_md_cic(R, Nf, L, Y.data(), nsub, a, out);
}

/* Poisson solve on the force mesh: the FFT part of Gravity::kick,
 * src/run/nbody.hh:103-110. `delta` holds the deposit (mean 1) on entry and
 * phi = G/a * IFFT(-FFT(delta-1)/k^2)/size on return. */
void oracle_poisson(int R, int N, double L, double G, double a, double *delta) {
    size_t size = ipow(N, R);
    std::vector<cplx> in(size), out(size);
    for (size_t i = 0; i < size; ++i) in[i] = delta[i] - 1.0;
    dft(in, out, R, N, FFTW_FORWARD);
    for (size_t i = 0; i < size; ++i) {
        double k[8];
        kvec(i, R, N, L, k);
        in[i] = out[i] * cplx(-1. / sqr(k, R));
    }
    in[0] = 0;
    dft(in, out, R, N, FFTW_BACKWARD);
    double s = (double)size / G * a;
    for (size_t i = 0; i < size; ++i) delta[i] = out[i].real() / s;
}

/* CIC interpolation of the finite-difference gradient of phi at X:
 * LinearInterpolation<Gradient<R>,R>::operator(), src/run/numeric.hh:6-45
 * over Gradient<R>::operator[], src/run/numeric.hh:72-103. Note the
 * unwrapped coordinate and the truncating cast (numeric.hh:19-29). */
void oracle_interp_gradient(int R, int N, double L, const double *phi, const double *X,
                            size_t n, double *out) {
    double res = L / N;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) {
        double x[8], A[2][8], v[8] = {0};
        int origin[8];
        for (int k = 0; k < R; ++k) {
            x[k] = X[i * R + k] / res;
            origin[k] = (int)(x[k]);
            A[1][k] = x[k] - origin[k];
            A[0][k] = 1 - A[1][k];
        }
        for (int j = 0; j < (1 << R); ++j) {
            double z = 1;
            int c[8];
            for (int k = 0; k < R; ++k) {
                int b = (j >> k) & 1;
                z *= A[b][k];
                c[k] = origin[k] + b;
            }
            size_t s = box_idx(c, R, N);
            int p0[8], q[8];
            decode(s, R, N, p0);
            double g[8];
            for (int k = 0; k < R; ++k) {
                size_t id[4];
                int off[4] = {-2, -1, 1, 2};
                for (int jj = 0; jj < 4; ++jj) {
                    std::memcpy(q, p0, sizeof(int) * R);
                    q[k] += off[jj];
                    id[jj] = box_idx(q, R, N);
                }
                double vv = phi[id[0]] / 12. - 2 * phi[id[1]] / 3. + 2 * phi[id[2]] / 3. -
                            phi[id[3]] / 12.;
                g[k] = vv / res;
            }
            for (int k = 0; k < R; ++k) v[k] += g[k] * z;
        }
        for (int k = 0; k < R; ++k) out[i * R + k] = v[k];
    }
}

/* Scale-factor rate adot(a) = H0 a sqrt(OL + Om a^-3 + Ok a^-2):
 * Cosmology::operator(), src/run/cosmology.hh:16-23. */
double oracle_adot(double H0, double Om, double OL, double a) {
    double Ok = 1 - Om - OL;
    return H0 * a * std::sqrt(OL + Om * std::pow(a, -3) + Ok * std::pow(a, -2));
}

/* One kick: deposit, Poisson, gather, momentum update. Gravity::kick,
 * src/run/nbody.hh:97-120. `phi_out` (optional, N^R) receives the potential. */
void oracle_kick(int R, int Nm, int f, double L, double H0, double Om, double OL, double *X,
                 double *P, double a, double da, double *phi_out) {
    int Nf = f * Nm;
    size_t np = ipow(Nm, R), nc = ipow(Nf, R);
    double mass = std::pow(double(Nf) / Nm, R);
    double G = 3. / 2 * Om * H0 * H0;
    std::vector<double> delta(nc), acc(np * R);
    oracle_md_cic(R, Nf, L, X, np, mass, delta.data());
    oracle_poisson(R, Nf, L, G, a, delta.data());
    double adot = oracle_adot(H0, Om, OL, a);
    oracle_interp_gradient(R, Nf, L, delta.data(), X, np, acc.data());
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < np; ++i)
        for (int k = 0; k < R; ++k) P[i * R + k] -= acc[i * R + k] * (da / adot);
    if (phi_out) std::memcpy(phi_out, delta.data(), nc * sizeof(double));
}

/* One drift: Gravity::drift, src/run/nbody.hh:122-133. */
void oracle_drift(int R, int Nm, double H0, double Om, double OL, double *X, const double *P,
                  double a, double da) {
    size_t np = ipow(Nm, R);
    double adot = oracle_adot(H0, Om, OL, a);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < np; ++i)
        for (int k = 0; k < R; ++k) X[i * R + k] += P[i * R + k] * (da / (a * a * adot));
}

/* Full leapfrog run: LeapFrog::run, src/run/leapfrog.hh:33-46, from the
 * potential on the mass mesh. On return X, P hold the final state. */
void oracle_run(int R, int Nm, int f, double L, double H0, double Om, double OL,
                const double *phi, double a0, double da, unsigned n, double *X, double *P) {
    oracle_zeldovich(R, Nm, L, phi, a0, a0 + da / 2, X, P);
    double a = a0;
    for (unsigned i = 0; i < n; ++i) {
        oracle_drift(R, Nm, H0, Om, OL, X, P, a, da);
        oracle_kick(R, Nm, f, L, H0, Om, OL, X, P, a + da / 2, da, nullptr);
        a += da;
    }
}

/* Shell-averaged power spectrum of a mesh (no reference counterpart in the
 * C++ tools; the estimator follows scripts/Power spectrum.ipynb: |FFT|^2
 * averaged by |k|). Bin j in 0..nbins-1 holds modes with
 * floor(|n| + 0.5) == j, |n| the integer wave-vector length; P is
 * |delta_hat|^2 * L^R / size^2 and k the mean |k| of the bin. */
void oracle_power_spectrum(int R, int N, double L, const double *delta, int nbins, double *k_out,
                           double *p_out, double *cnt_out) {
    size_t size = ipow(N, R);
    std::vector<cplx> in(size), out(size);
    for (size_t i = 0; i < size; ++i) in[i] = delta[i];
    dft(in, out, R, N, FFTW_FORWARD);
    std::vector<double> ps(nbins, 0), ks(nbins, 0), cn(nbins, 0);
    for (size_t i = 0; i < size; ++i) {
        int x[8];
        decode(i, R, N, x);
        long n2 = 0;
        for (int k = 0; k < R; ++k) {
            long s = x[k] > N / 2 ? x[k] - N : x[k];
            n2 += s * s;
        }
        double nn = std::sqrt((double)n2);
        int b = (int)std::floor(nn + 0.5);
        if (b < nbins) {
            ps[b] += std::norm(out[i]);
            ks[b] += nn * 2 * M_PI / L;
            cn[b] += 1;
        }
    }
    double norm = std::pow(L, R) / ((double)size * (double)size);
    for (int b = 0; b < nbins; ++b) {
        cnt_out[b] = cn[b];
        k_out[b] = cn[b] > 0 ? ks[b] / cn[b] : 0;
        p_out[b] = cn[b] > 0 ? ps[b] / cn[b] * norm : 0;
    }
}

}  // extern "C"

/* ------------------------------------------------------------------------
 * FP64 CPU adjoint of the differentiable model (no reference counterpart:
 * the reference has no adjoint). Forward: white noise w -> scale-free GRF
 * (oracle_grf_scale_free) -> potential (oracle_potential) -> Zel'dovich
 * (oracle_zeldovich) -> n leapfrog steps (oracle_drift / oracle_kick) ->
 * final CIC density (oracle_md_cic - 1). The adjoint is derived directly in
 * the reference's physical units (absolute X, momentum P), keeping every
 * forward state in memory (small test sizes only).
 * ---------------------------------------------------------------------- */
namespace {

struct DiffCfg {
    int R, mbits, f;
    double L, ns, scale, sigma, H0, Om, OL, a0, da;
    int smooth;
    unsigned n;
};

/* Linear Fourier operator on an R-cube: out = Re IFFT(FFT(in) * mult) / size,
 * mult(idx) given, DC forced to zero. */
template <typename M>
void fourier_op(int R, int N, const double *in, double *out, M mult) {
    size_t size = ipow(N, R);
    std::vector<cplx> a(size), b(size);
    for (size_t i = 0; i < size; ++i) a[i] = in[i];
    dft(a, b, R, N, FFTW_FORWARD);
    for (size_t i = 0; i < size; ++i) a[i] = b[i] * mult(i);
    a[0] = 0;
    dft(a, b, R, N, FFTW_BACKWARD);
    for (size_t i = 0; i < size; ++i) out[i] = b[i].real() / (double)size;
}

/* dW_b/dx_k for CIC weights with A0 = 1 - A1. */
double dW(const double *A0, const double *A1, int R, int b, int k) {
    double z = ((b >> k) & 1) ? 1.0 : -1.0;
    for (int l = 0; l < R; ++l)
        if (l != k) z *= ((b >> l) & 1) ? A1[l] : A0[l];
    return z;
}

/* -sum_k FD4_k(U_k) / res on an R-cube (the adjoint of the FD4 gradient). */
void neg_div(int R, int N, double res, const std::vector<std::vector<double>> &U, double *out) {
    size_t size = ipow(N, R);
#pragma omp parallel for schedule(static)
    for (size_t x = 0; x < size; ++x) {
        int p0[8], q[8];
        decode(x, R, N, p0);
        double acc = 0;
        for (int k = 0; k < R; ++k) {
            size_t id[4];
            int off[4] = {-2, -1, 1, 2};
            for (int j = 0; j < 4; ++j) {
                std::memcpy(q, p0, sizeof(int) * R);
                q[k] += off[j];
                id[j] = box_idx(q, R, N);
            }
            const std::vector<double> &u = U[k];
            acc += u[id[0]] / 12. - 2 * u[id[1]] / 3. + 2 * u[id[2]] / 3. - u[id[3]] / 12.;
        }
        out[x] = -acc / res;
    }
}

}  // namespace

extern "C" {

/* noisebar = dL/dw for L with dL/d(final density) = deltabar. Also writes
 * the final density into delta_out (may be NULL). */
void oracle_diff_adjoint(int R, int mbits, int f, double L, double ns, int smooth, double scale, double sigma,
                         double H0, double Om, double OL, double a0, double da, unsigned n, const double *w,
                         const double *deltabar, double *delta_out, double *noisebar) {
    const int Nm = 1 << mbits, Nf = Nm * f;
    const size_t np = ipow(Nm, R), nc = ipow(Nf, R);
    const double res_f = L / Nf, res_m = L / Nm, mass = std::pow((double)Nf / Nm, R);
    const double Gc = 3. / 2 * Om * H0 * H0;
    /* ---- forward, keeping states ---- */
    std::vector<double> dens(np), phim(np);
    oracle_grf_scale_free(R, mbits, L, ns, smooth, scale, sigma, w, dens.data());
    phim = dens;
    oracle_potential(R, mbits, L, phim.data());
    std::vector<double> X(np * R), P(np * R);
    double a_pos = a0, a_mom = a0 + da / 2;
    oracle_zeldovich(R, Nm, L, phim.data(), a_pos, a_mom, X.data(), P.data());
    std::vector<std::vector<double>> Xs(n), phis(n);  // positions at the kicks and their potentials
    std::vector<double> as(n);
    double a = a0;
    for (unsigned i = 0; i < n; ++i) {
        as[i] = a;
        oracle_drift(R, Nm, H0, Om, OL, X.data(), P.data(), a, da);
        Xs[i] = X;
        phis[i].resize(nc);
        oracle_kick(R, Nm, f, L, H0, Om, OL, X.data(), P.data(), a + da / 2, da, phis[i].data());
        a += da;
    }
    std::vector<double> dfin(nc);
    oracle_md_cic(R, Nf, L, X.data(), np, mass, dfin.data());
    if (delta_out)
        for (size_t c = 0; c < nc; ++c) delta_out[c] = dfin[c] - 1.0;

    /* deposit-weight frame of a particle: cells and weights of md_cic */
    auto dep_frame = [&](const double *x, int *origin, double *A0, double *A1) {
        for (int k = 0; k < R; ++k) {
            double p0 = dmod(x[k], L) / res_f;
            origin[k] = (int)p0;
            A1[k] = p0 - origin[k];
            A0[k] = 1 - A1[k];
        }
    };
    auto gat_frame = [&](const double *x, int *origin, double *A0, double *A1) {
        for (int k = 0; k < R; ++k) {
            double xx = x[k] / res_f;
            origin[k] = (int)xx;
            A1[k] = xx - origin[k];
            A0[k] = 1 - A1[k];
        }
    };
    auto corner = [&](const int *origin, int b) {
        int c[8];
        for (int k = 0; k < R; ++k) c[k] = origin[k] + ((b >> k) & 1);
        return box_idx(c, R, Nf);
    };
    auto poisson_op = [&](const double *in, double *out, double am) {
        fourier_op(R, Nf, in, out, [&](size_t i) {
            double k[8];
            kvec(i, R, Nf, L, k);
            return cplx(-1. / sqr(k, R) * Gc / am);
        });
    };

    /* ---- backward ---- */
    std::vector<double> Xb(np * R, 0.0), Pb(np * R, 0.0);
#pragma omp parallel for schedule(static)
    for (size_t j = 0; j < np; ++j) {  // through the final deposit
        int o[8];
        double A0[8], A1[8];
        dep_frame(&X[j * R], o, A0, A1);
        for (int b = 0; b < (1 << R); ++b) {
            double v = deltabar[corner(o, b)];
            for (int k = 0; k < R; ++k) Xb[j * R + k] += mass * dW(A0, A1, R, b, k) * v / res_f;
        }
    }
    for (int i = (int)n - 1; i >= 0; --i) {
        const double am = as[i] + da / 2;
        const double ckp = da / oracle_adot(H0, Om, OL, am);
        const double cdp = da / (as[i] * as[i] * oracle_adot(H0, Om, OL, as[i]));
        const std::vector<double> &Xk = Xs[i];
        const std::vector<double> &phi = phis[i];
        std::vector<double> g(nc * R);
        oracle_gradient(R, Nf, L, phi.data(), g.data());  // physical gradient at the nodes
        const std::vector<double> v = Pb;
        // U_k = gather-transpose deposit of v_k
        std::vector<std::vector<double>> U(R, std::vector<double>(nc, 0.0));
        for (size_t j = 0; j < np; ++j) {
            int o[8];
            double A0[8], A1[8];
            gat_frame(&Xk[j * R], o, A0, A1);
            for (int b = 0; b < (1 << R); ++b) {
                double z = 1;
                for (int k = 0; k < R; ++k) z *= ((b >> k) & 1) ? A1[k] : A0[k];
                size_t c = corner(o, b);
                for (int k = 0; k < R; ++k) U[k][c] += v[j * R + k] * z;
            }
        }
        std::vector<double> div(nc), rhob(nc);
        neg_div(R, Nf, res_f, U, div.data());
        poisson_op(div.data(), rhob.data(), am);
#pragma omp parallel for schedule(static)
        for (size_t j = 0; j < np; ++j) {
            double t1[8] = {0}, t2[8] = {0};
            int o[8];
            double A0[8], A1[8];
            gat_frame(&Xk[j * R], o, A0, A1);
            for (int b = 0; b < (1 << R); ++b) {
                size_t c = corner(o, b);
                double vg = 0;
                for (int k = 0; k < R; ++k) vg += v[j * R + k] * g[c * R + k];
                for (int k = 0; k < R; ++k) t1[k] += dW(A0, A1, R, b, k) * vg / res_f;
            }
            dep_frame(&Xk[j * R], o, A0, A1);
            for (int b = 0; b < (1 << R); ++b) {
                double r = rhob[corner(o, b)];
                for (int k = 0; k < R; ++k) t2[k] += mass * dW(A0, A1, R, b, k) * r / res_f;
            }
            for (int k = 0; k < R; ++k) {
                double xb = Xb[j * R + k] - ckp * (t1[k] + t2[k]);
                Xb[j * R + k] = xb;
                Pb[j * R + k] = v[j * R + k] + cdp * xb;
            }
        }
    }
    /* Zel'dovich: X = q - a_pos u, P = -a_mom u, u = FD4(phi_m)/res_m */
    std::vector<std::vector<double>> ub(R, std::vector<double>(np));
    for (size_t j = 0; j < np; ++j)
        for (int k = 0; k < R; ++k) ub[k][j] = -a_pos * Xb[j * R + k] - a_mom * Pb[j * R + k];
    std::vector<double> phib(np), densb(np);
    neg_div(R, Nm, res_m, ub, phib.data());
    /* potential operator (symmetric): -1/k^2 physical, DC 0 */
    fourier_op(R, Nm, phib.data(), densb.data(), [&](size_t i) {
        double k[8];
        kvec(i, R, Nm, L, k);
        return cplx(-1. / sqr(k, R));
    });
    /* random field: dens = s y, y = L_F w, var = |L_PS w|^2 / N, s = sigma/sqrt(var) */
    const double t = scale * Nm / L;
    auto PSf = [&](size_t i, bool with_s) {
        double k[8];
        kvec(i, R, Nm, (double)Nm, k);
        double p = std::sqrt(std::pow(std::sqrt(sqr(k, R)), ns));
        return with_s ? p * scale_filter(k, R, t) : p;
    };
    std::vector<double> y(np), z(np), q(np), lfd(np);
    fourier_op(R, Nm, w, y.data(), [&](size_t i) { return cplx(PSf(i, smooth != 0)); });
    fourier_op(R, Nm, w, z.data(), [&](size_t i) { return cplx(PSf(i, true)); });
    fourier_op(R, Nm, z.data(), q.data(), [&](size_t i) { return cplx(PSf(i, true)); });
    fourier_op(R, Nm, densb.data(), lfd.data(), [&](size_t i) { return cplx(PSf(i, smooth != 0)); });
    double var = 0, dot = 0;
    for (size_t j = 0; j < np; ++j) {
        var += z[j] * z[j];
        dot += y[j] * densb[j];
    }
    var /= (double)np;
    const double s = sigma / std::sqrt(var);
    for (size_t j = 0; j < np; ++j) noisebar[j] = s * lfd[j] - (s / var) * dot / (double)np * q[j];
}

/* The forward model alone: final CIC density contrast from the noise. */
void oracle_diff_forward(int R, int mbits, int f, double L, double ns, int smooth, double scale, double sigma,
                         double H0, double Om, double OL, double a0, double da, unsigned n, const double *w,
                         double *delta_out) {
    const int Nm = 1 << mbits, Nf = Nm * f;
    const size_t np = ipow(Nm, R), nc = ipow(Nf, R);
    std::vector<double> dens(np);
    oracle_grf_scale_free(R, mbits, L, ns, smooth, scale, sigma, w, dens.data());
    oracle_potential(R, mbits, L, dens.data());
    std::vector<double> X(np * R), P(np * R);
    oracle_run(R, Nm, f, L, H0, Om, OL, dens.data(), a0, da, n, X.data(), P.data());
    oracle_md_cic(R, Nf, L, X.data(), np, std::pow((double)Nf / Nm, R), delta_out);
    for (size_t c = 0; c < nc; ++c) delta_out[c] -= 1.0;
}

/* Friends-of-friends tags, fof_run<R> (src/fof/fof.cc:164-231): for every
 * particle in index order that has no tag yet, a flood fill with a stack
 * (flood_fill, src/fof/fof.cc:17-40) paints the particles reachable through
 * friends with the next group number. Friends: Proximity (src/fof/fof.cc:
 * 71-99), the raw difference wrapped once per axis, d.sqr() <= ll * ll. The
 * reference finds the candidates with a kd-tree (src/fof/kdtree.hh) whose box
 * test prunes only boxes that cannot hold a friend; here a cell list with
 * cells no smaller than ll (all pairs when L / ll < 3) gives the same set.
 * Returns the number of groups. */
unsigned long long oracle_fof(int R, size_t n, double L, double ll, const double *X, unsigned long long *tags) {
    long long nc = (long long)(L / (ll * (1.0 + 1e-9)));
    while (nc > 3 && (double)ipow((size_t)nc, R) > 4.0 * (double)n + 64.0) --nc;
    if (nc < 3) nc = 1;
    const size_t cells = ipow((size_t)nc, R);
    std::vector<size_t> head(cells, (size_t)-1), next(n);
    std::vector<int> cc(n * R);
    for (size_t i = n; i-- > 0;) {
        size_t id = 0;
        for (int k = R - 1; k >= 0; --k) {
            double w = X[i * R + k] - std::floor(X[i * R + k] / L) * L;
            long long c = (long long)(w * ((double)nc / L));
            c = c < 0 ? 0 : (c >= nc ? nc - 1 : c);
            cc[i * R + k] = (int)c;
            id = id * (size_t)nc + (size_t)c;
        }
        next[i] = head[id];
        head[id] = i;
    }
    const double half = L / 2, rsqr = ll * ll;
    auto friends = [&](size_t a, size_t b) {
        double v = 0;
        for (int k = 0; k < R; ++k) {
            double e = X[b * R + k] - X[a * R + k], d;
            if (e > half) d = e - L;
            else if (e < -half) d = e + L;
            else d = e;
            v += d * d;
        }
        return v <= rsqr;
    };
    for (size_t i = 0; i < n; ++i) tags[i] = 0;
    unsigned long long current = 1;
    std::vector<size_t> stack;
    const int nb = nc == 1 ? 1 : (R == 2 ? 9 : 27);
    for (size_t start = 0; start < n; ++start) {
        if (tags[start] != 0) continue;
        tags[start] = current;
        stack.push_back(start);
        while (!stack.empty()) {
            size_t a = stack.back();
            stack.pop_back();
            for (int q = 0; q < nb; ++q) {
                size_t id = 0;
                for (int k = R - 1; k >= 0; --k) {
                    long long c = cc[a * R + k] + (nb == 1 ? 0 : (q / (k == 0 ? 1 : k == 1 ? 3 : 9)) % 3 - 1);
                    c = c < 0 ? c + nc : (c >= nc ? c - nc : c);
                    id = id * (size_t)nc + (size_t)c;
                }
                for (size_t b = head[id]; b != (size_t)-1; b = next[b]) {
                    if (tags[b] == current || !friends(a, b)) continue;
                    tags[b] = current;
                    stack.push_back(b);
                }
            }
        }
        ++current;
    }
    return current - 1;
}

}  // extern "C"
