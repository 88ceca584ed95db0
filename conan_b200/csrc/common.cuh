// common.cuh -- error state, geometry, RNG and reduction helpers shared by the
// kernels of libconan_pm.so.
#pragma once

#include <cuda.h>  // CUtensorMap (the encoder is fetched from the driver at run time)
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>

#include "../../include/conan_pm.h"

namespace conan {

// ---------------------------------------------------------------- errors --

// Per-thread message of the last failed call (conan_last_error()).
std::string &last_error();
int set_error(int code, const char *fmt, ...);

#define CONAN_CUDA(call)                                                              \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess)                                                        \
            return ::conan::set_error(CONAN_ERR_CUDA, "%s failed: %s (%s:%d)", #call, \
                                      cudaGetErrorString(e_), __FILE__, __LINE__);    \
    } while (0)

#define CONAN_CUFFT(call)                                                                 \
    do {                                                                                  \
        cufftResult r_ = (call);                                                          \
        if (r_ != CUFFT_SUCCESS)                                                          \
            return ::conan::set_error(CONAN_ERR_CUDA, "%s failed: cufft error %d (%s:%d)", \
                                      #call, (int)r_, __FILE__, __LINE__);                \
    } while (0)

#define CONAN_TRY(call)             \
    do {                            \
        int rc_ = (call);           \
        if (rc_ != CONAN_OK) return rc_; \
    } while (0)

// Launch-error check after a kernel launch.
#define CONAN_LAUNCHED()                                                                   \
    do {                                                                                   \
        cudaError_t e_ = cudaGetLastError();                                               \
        if (e_ != cudaSuccess)                                                             \
            return ::conan::set_error(CONAN_ERR_CUDA, "kernel launch failed: %s (%s:%d)",  \
                                      cudaGetErrorString(e_), __FILE__, __LINE__);         \
    } while (0)

// Raises (never lowers) kernel kern's limit of dynamic shared memory to at
// least `bytes`. The limit belongs to the kernel function, not to a handle:
// lowering it for one handle's launch configuration would make another
// handle's larger launch of the same kernel fail. False when the device
// cannot give that much (the error state is cleared).
template <typename K> bool raise_dyn_smem(K kern, size_t bytes) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if ((size_t)fa.maxDynamicSharedSizeBytes >= bytes) return true;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}

inline bool is_pow2(long long n) { return n > 0 && (n & (n - 1)) == 0; }
inline int ilog2(long long n) {
    int s = 0;
    while ((1LL << s) < n) ++s;
    return s;
}

// -------------------------------------------------------------- geometry --

// A batch of `batch` periodic meshes of n^R cells each, axis 0 fastest (the
// reference's Box<R>, src/base/box.hh:26-82), stored back to back, and their
// half-complex spectra of nh x n^(R-1) values each, nh = n/2 + 1, as cuFFT
// lays out an R2C transform whose fastest axis is 0. Global cell index =
// member << cshift | local index; `cells` and `spec` count the whole batch.
struct Mesh {
    int R;
    int n;       // cells per side
    int shift;   // log2(n)
    size_t cells;
    int nh;      // n/2 + 1
    size_t spec; // batch * nh * n^(R-1)
    int cshift;  // R * shift: log2 of the cells of one member
    size_t mspec;  // nh * n^(R-1): spectrum values of one member
    int batch;
    double inv_nh;  // 1 / nh, for the quotient of half-spectrum indices
};

inline Mesh make_mesh(int R, int n, int batch = 1) {
    Mesh m;
    m.R = R;
    m.n = n;
    m.shift = ilog2(n);
    m.cshift = R * m.shift;
    m.batch = batch;
    m.cells = (size_t)batch << m.cshift;
    m.nh = n / 2 + 1;
    m.mspec = (size_t)m.nh;
    for (int i = 1; i < R; ++i) m.mspec *= (size_t)n;
    m.spec = m.mspec * (size_t)batch;
    m.inv_nh = 1.0 / (double)m.nh;
    return m;
}

// First global cell of the member owning global cell / spectrum element.
__host__ __device__ inline size_t member_cells(const Mesh &m, size_t member) { return member << m.cshift; }

// Signed integer wave number of index i on an n-mesh; index n/2 keeps the
// positive sign like Fourier::kspace (src/base/fourier.hh:42-55).
__host__ __device__ inline int wave_index(int i, int n) { return i > n / 2 ? i - n : i; }

// Squared integer wave-vector length of half-spectrum element e (of any
// member of the batch).
__device__ inline long long spec_k2(size_t e, const Mesh &m, int *kv) {
    // row = e / nh from the double reciprocal (exact after one correction:
    // e < 2^53); the row's low (R-1) shift bits are the member's y, z
    // indices, the bits above them the member (ignored)
    size_t rest = (size_t)((double)e * m.inv_nh);
    long long kr = (long long)e - (long long)rest * m.nh;
    if (kr < 0) {
        --rest;
        kr += m.nh;
    } else if (kr >= m.nh) {
        ++rest;
        kr -= m.nh;
    }
    int kx = (int)kr;
    long long s = (long long)kx * kx;
    kv[0] = kx;
    for (int a = 1; a < m.R; ++a) {
        int ia = (int)(rest & (size_t)(m.n - 1));
        rest >>= m.shift;
        int w = wave_index(ia, m.n);
        kv[a] = w;
        s += (long long)w * w;
    }
    return s;
}

// Number of full-spectrum modes a half-spectrum element stands for: the
// kx = 0 and kx = n/2 planes are their own mirrors.
__device__ inline double spec_weight(int kx, int n) { return (kx == 0 || kx == n / 2) ? 1.0 : 2.0; }

// ------------------------------------------------------------ complex ---

template <typename T> struct Cplx;
template <> struct Cplx<float> { typedef cufftComplex type; };
template <> struct Cplx<double> { typedef cufftDoubleComplex type; };

// ------------------------------------------------------------ Philox RNG --

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11), with the round
// multipliers and Weyl key increments published there.
__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c[0];
        uint64_t p1 = (uint64_t)M1 * c[2];
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += W0;
        k1 += W1;
    }
}

// Two unit normals for pair index j of the stream `seed` (Box-Muller on two
// 53-bit uniforms in (0,1)). Cells 2j and 2j+1 of a noise field take them.
__device__ inline void philox_normal_pair(unsigned long long seed, unsigned long long j,
                                          double *z0, double *z1) {
    uint32_t c[4] = {(uint32_t)j, (uint32_t)(j >> 32), 0x636f6e61u /* stream tag */, 0u};
    philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
    unsigned long long a = (((unsigned long long)c[0] << 32) | c[1]) >> 11;
    unsigned long long b = (((unsigned long long)c[2] << 32) | c[3]) >> 11;
    double u1 = ((double)a + 0.5) * 0x1p-53;
    double u2 = ((double)b + 0.5) * 0x1p-53;
    double r = sqrt(-2.0 * log(u1));
    double s, co;
    sincospi(2.0 * u2, &s, &co);
    *z0 = r * co;
    *z1 = r * s;
}

// ------------------------------------------------- deterministic sums --

// Fixed-pattern warp sum (same order on every run).
template <typename T> __device__ inline T warp_sum(T v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-pattern block sum for blockDim.x a multiple of 32 (<= 1024); the
// result is valid in thread 0.
template <typename T> __device__ inline T block_sum(T v) {
    __shared__ T part[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) part[w] = v;
    __syncthreads();
    T r = 0;
    if (w == 0) {
        int nw = (blockDim.x + 31) >> 5;
        r = lane < nw ? part[lane] : T(0);
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

}  // namespace conan
