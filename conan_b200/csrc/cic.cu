// cic.cu -- the `cic` tool on the GPU: the density of a snapshot on an
// Eulerian mesh, cic_run<R> (src/cic/cic.hh:49-81), optionally from a
// sub-sampled Lagrangian grid whose positions are interpolated from the
// particles' displacements.
//
// Positions and weights are FP64 with the reference's arithmetic (its
// truncating floating modulus, its corner order); each corner weight is
// rounded to a multiple of 2^-40 and summed as a 64-bit integer, so the mesh
// does not depend on the order of the atomic adds (the reference sums in an
// OpenMP critical section, in thread order).
#include <cmath>

#include "pm.cuh"

namespace conan {
namespace {

constexpr double CIC_UNIT = 1099511627776.0;  // 2^40

// modulus(double, double), src/base/misc.hh:144-148.
__device__ inline double ref_dmod(double a, double b) {
    if (a < 0) return a - (double)static_cast<int>(a / b - 1) * b;
    return a - (double)static_cast<int>(a / b) * b;
}

struct CicMesh {
    int nf, shift;  // Eulerian cells per side, log2
    double L, res;  // box size, Eulerian cell size (L / nf)
};

// md_cic_T's inner loop (src/cic/cic.hh:14-38) for one position, weights
// without the mass (applied to the sums).
template <int R>
__device__ inline void cic_add(const double *x, const CicMesh &m, unsigned long long *__restrict__ acc) {
    double A[2][3];
    int o[3];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const double p0 = ref_dmod(x[k], m.L) / m.res;
        o[k] = (int)p0;
        A[1][k] = p0 - o[k];
        A[0][k] = 1 - A[1][k];
    }
    const unsigned mask = (unsigned)m.nf - 1;
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        double z = 1;
        size_t idx = 0;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int bk = (b >> k) & 1;
            z *= A[bk][k];
            idx |= (size_t)((unsigned)(o[k] + bk) & mask) << (k * m.shift);
        }
        const unsigned long long q = __double2ull_rn(z * CIC_UNIT);
        if (q) atomicAdd(acc + idx, q);
    }
}

template <int R>
__global__ void __launch_bounds__(256) k_cic_particles(const double *__restrict__ X, size_t n, CicMesh m,
                                                       unsigned long long *__restrict__ acc) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x[3];
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = X[i * R + k];
    cic_add<R>(x, m, acc);
}

// Sub-sampled positions (src/cic/cic.hh:62-74): grid point y of the (s N)^R
// grid plus the linear interpolation (LinearInterpolation, src/run/numeric.hh:
// 17-42) of the displacement field D = X - q on the mass grid.
template <int R>
__global__ void __launch_bounds__(256) k_cic_subsample(const double *__restrict__ D, int nm, int mshift,
                                                       int ns, int sshift, double dy, double res_m, CicMesh m,
                                                       unsigned long long *__restrict__ acc) {
    const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ((size_t)1 << (R * sshift))) return;
    double y[3], A[2][3];
    int o[3];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int jk = (int)((j >> (k * sshift)) & (size_t)(ns - 1));
        y[k] = (double)jk * dy;
        const double xk = y[k] / res_m;
        o[k] = (int)xk;
        A[1][k] = xk - o[k];
        A[0][k] = 1 - A[1][k];
    }
    double v[3] = {0, 0, 0};
    const unsigned mmask = (unsigned)nm - 1;
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        double z = 1;
        size_t id = 0;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const int bk = (b >> k) & 1;
            z *= A[bk][k];
            id |= (size_t)((unsigned)(o[k] + bk) & mmask) << (k * mshift);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) v[k] += D[id * R + k] * z;
    }
    double x[3];
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = y[k] + v[k];
    cic_add<R>(x, m, acc);
}

// D = X - G on the mass grid (src/cic/cic.hh:65-66), G = grid_space(N, L).
template <int R>
__global__ void k_cic_displacement(const double *__restrict__ X, double *__restrict__ D, int nm, int mshift,
                                   double dq) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ((size_t)1 << (R * mshift))) return;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int qk = (int)((i >> (k * mshift)) & (size_t)(nm - 1));
        D[i * R + k] = X[i * R + k] - (double)qk * dq;
    }
}

__global__ void k_cic_finish(const unsigned long long *__restrict__ acc, double *__restrict__ rho, size_t n,
                             double scale) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rho[i] = (double)acc[i] * scale;
}

template <int R>
int cic_run(const conan_cic_params &p, const double *Xh, double *rho_h) {
    const int N = p.n_mass, Nf = p.n_mass * p.f, s = p.sub_sample;
    const size_t np = (size_t)1 << (R * ilog2(N)), nc = (size_t)1 << (R * ilog2(Nf));
    CicMesh m{Nf, ilog2(Nf), p.size, p.size / Nf};
    cudaStream_t st = nullptr;
    double *X = nullptr, *D = nullptr, *rho = nullptr;
    unsigned long long *acc = nullptr;
    int rc = CONAN_OK;
    auto fail = [&](cudaError_t e, const char *what) {
        if (rc == CONAN_OK && e != cudaSuccess) {
            cudaGetLastError();
            rc = set_error(e == cudaErrorMemoryAllocation ? CONAN_ERR_ALLOC : CONAN_ERR_CUDA, "conan_cic: %s: %s", what,
                           cudaGetErrorString(e));
        }
        return rc == CONAN_OK;
    };
    if (fail(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream") &&
        fail(cudaMalloc(&X, np * R * sizeof(double)), "cudaMalloc") &&
        fail(cudaMalloc(&acc, nc * sizeof(unsigned long long)), "cudaMalloc") &&
        fail(cudaMalloc(&rho, nc * sizeof(double)), "cudaMalloc") &&
        fail(cudaMemcpyAsync(X, Xh, np * R * sizeof(double), cudaMemcpyHostToDevice, st), "copy") &&
        fail(cudaMemsetAsync(acc, 0, nc * sizeof(unsigned long long), st), "memset")) {
        double mass = 1.0;
        if (s == 1) {
            k_cic_particles<R><<<(unsigned)((np + 255) / 256), 256, 0, st>>>(X, np, m, acc);
            fail(cudaGetLastError(), "k_cic_particles");
        } else if (fail(cudaMalloc(&D, np * R * sizeof(double)), "cudaMalloc")) {
            const int ns = N * s;
            const size_t nsub = (size_t)1 << (R * ilog2(ns));
            k_cic_displacement<R><<<(unsigned)((np + 255) / 256), 256, 0, st>>>(X, D, N, ilog2(N), p.size / N);
            fail(cudaGetLastError(), "k_cic_displacement");
            k_cic_subsample<R><<<(unsigned)((nsub + 255) / 256), 256, 0, st>>>(
                D, N, ilog2(N), ns, ilog2(ns), p.size / ns, p.size / N, m, acc);
            fail(cudaGetLastError(), "k_cic_subsample");
            mass = std::pow(double(s * N) / double(Nf), -float(R));  // src/cic/cic.hh:76
        }
        if (rc == CONAN_OK) {
            k_cic_finish<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(acc, rho, nc, mass / CIC_UNIT);
            fail(cudaGetLastError(), "k_cic_finish");
        }
        if (rc == CONAN_OK) fail(cudaMemcpyAsync(rho_h, rho, nc * sizeof(double), cudaMemcpyDeviceToHost, st), "copy");
        if (rc == CONAN_OK) fail(cudaStreamSynchronize(st), "run");
    }
    if (st) cudaStreamSynchronize(st);
    cudaFree(X);
    cudaFree(D);
    cudaFree(acc);
    cudaFree(rho);
    if (st) cudaStreamDestroy(st);
    return rc;
}

}  // namespace
}  // namespace conan

using namespace conan;

extern "C" int conan_cic(const conan_cic_params *p, const double *X, double *rho_out) {
    if (!p) return set_error(CONAN_ERR_ARG, "null parameters");
    if (p->dim < 1 || p->dim > 3) return set_error(CONAN_ERR_UNSUPPORTED, "conan_cic: dim = %d (1..3)", p->dim);
    if (p->n_mass < 2 || !is_pow2(p->n_mass) || p->f < 1 || !is_pow2(p->f) || p->sub_sample < 1 ||
        !is_pow2(p->sub_sample))
        return set_error(CONAN_ERR_ARG, "conan_cic: n_mass, f and sub_sample must be powers of two");
    if (!(p->size > 0)) return set_error(CONAN_ERR_ARG, "conan_cic: box size must be positive");
    long long cells = 1, sub = 1;
    for (int k = 0; k < p->dim; ++k) {
        cells *= (long long)p->n_mass * p->f;
        sub *= (long long)p->n_mass * p->sub_sample;
    }
    if (cells >= (1LL << 32) || sub >= (1LL << 32))
        return set_error(CONAN_ERR_ARG, "conan_cic: mesh or sub-sampled grid beyond 2^32 points");
    if (!X || !rho_out) return set_error(CONAN_ERR_ARG, "conan_cic: null positions or output");
    CONAN_TRY(device_guard(p->device));
    switch (p->dim) {
        case 1: return cic_run<1>(*p, X, rho_out);
        case 2: return cic_run<2>(*p, X, rho_out);
        default: return cic_run<3>(*p, X, rho_out);
    }
}
