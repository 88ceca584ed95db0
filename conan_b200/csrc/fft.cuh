// fft.cuh -- cuFFT real<->half-complex plans over the cubic meshes of Mesh.
#pragma once

#include "common.cuh"

namespace conan {

// R2C / C2R pair for `batch` meshes of n^R cells stored back to back
// (real stride n^R, spectrum stride nh*n^(R-1)). Axis 0 is the fastest axis
// of both the real mesh and the half-complex spectrum. The work area is
// supplied by the owner so several plans can share one buffer.
struct FFTPair {
    cufftHandle r2c = 0, c2r = 0;
    size_t work_bytes = 0;
    bool dbl = false;

    int create(const Mesh &m, bool is_double, int batch) {
        dbl = is_double;
        int n[3];
        for (int i = 0; i < m.R; ++i) n[i] = m.n;  // cubic: slowest..fastest all n
        long long real_dist = 1LL << m.cshift, cplx_dist = (long long)m.mspec;
        size_t w1 = 0, w2 = 0;
        CONAN_CUFFT(cufftCreate(&r2c));
        CONAN_CUFFT(cufftCreate(&c2r));
        CONAN_CUFFT(cufftSetAutoAllocation(r2c, 0));
        CONAN_CUFFT(cufftSetAutoAllocation(c2r, 0));
        CONAN_CUFFT(cufftMakePlanMany(r2c, m.R, n, nullptr, 1, (int)real_dist, nullptr, 1,
                                      (int)cplx_dist, dbl ? CUFFT_D2Z : CUFFT_R2C, batch, &w1));
        CONAN_CUFFT(cufftMakePlanMany(c2r, m.R, n, nullptr, 1, (int)cplx_dist, nullptr, 1,
                                      (int)real_dist, dbl ? CUFFT_Z2D : CUFFT_C2R, batch, &w2));
        work_bytes = w1 > w2 ? w1 : w2;
        return CONAN_OK;
    }
    // 2D transforms of every z plane (3D meshes): the same half-spectrum
    // layout as the 3D pair with z left in real space.
    int create_planes(const Mesh &m, bool is_double, int batch) {
        dbl = is_double;
        int n[2] = {m.n, m.n};
        long long real_dist = (long long)m.n * m.n, cplx_dist = (long long)m.n * m.nh;
        const int planes = batch * m.n;
        size_t w1 = 0, w2 = 0;
        CONAN_CUFFT(cufftCreate(&r2c));
        CONAN_CUFFT(cufftCreate(&c2r));
        CONAN_CUFFT(cufftSetAutoAllocation(r2c, 0));
        CONAN_CUFFT(cufftSetAutoAllocation(c2r, 0));
        CONAN_CUFFT(cufftMakePlanMany(r2c, 2, n, nullptr, 1, (int)real_dist, nullptr, 1, (int)cplx_dist,
                                      dbl ? CUFFT_D2Z : CUFFT_R2C, planes, &w1));
        CONAN_CUFFT(cufftMakePlanMany(c2r, 2, n, nullptr, 1, (int)cplx_dist, nullptr, 1, (int)real_dist,
                                      dbl ? CUFFT_Z2D : CUFFT_C2R, planes, &w2));
        work_bytes = w1 > w2 ? w1 : w2;
        return CONAN_OK;
    }
    int bind(void *work, cudaStream_t s) {
        CONAN_CUFFT(cufftSetWorkArea(r2c, work));
        CONAN_CUFFT(cufftSetWorkArea(c2r, work));
        CONAN_CUFFT(cufftSetStream(r2c, s));
        CONAN_CUFFT(cufftSetStream(c2r, s));
        return CONAN_OK;
    }
    void destroy() {
        if (r2c) cufftDestroy(r2c);
        if (c2r) cufftDestroy(c2r);
        r2c = c2r = 0;
    }
    int forward(float *in, cufftComplex *out) {
        CONAN_CUFFT(cufftExecR2C(r2c, in, out));
        return CONAN_OK;
    }
    int forward(double *in, cufftDoubleComplex *out) {
        CONAN_CUFFT(cufftExecD2Z(r2c, in, out));
        return CONAN_OK;
    }
    // Unnormalised inverse; overwrites `in`.
    int inverse(cufftComplex *in, float *out) {
        CONAN_CUFFT(cufftExecC2R(c2r, in, out));
        return CONAN_OK;
    }
    int inverse(cufftDoubleComplex *in, double *out) {
        CONAN_CUFFT(cufftExecZ2D(c2r, in, out));
        return CONAN_OK;
    }
};

}  // namespace conan
