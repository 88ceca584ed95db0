// ic.cuh -- device-side building blocks of the initial conditions, shared by
// the ic entry points, the differentiable model and the ensemble.
#pragma once

#include "common.cuh"
#include "fft.cuh"

namespace conan {

enum { IC_SCALE_FREE = 0, IC_CDM = 1 };

struct ICFilter {
    int mode;
    double ns;      // spectral slope
    double t;       // Fourier::scale parameter, scale * N / L (cells)
    double L;       // box size
    double Omega0;  // CDM branch
    double h;       // H0 / 100 (CDM branch)
};

int check_ic_params(const conan_ic_params *p);

// Philox white noise into a device mesh.
template <typename T> int noise_device(const Mesh &m, unsigned long long seed, T *mesh, cudaStream_t st);
// Noise mesh -> density mesh, in place (uses spec as scratch).
template <typename T>
int grf_device(const conan_ic_params &p, const Mesh &m, T *mesh, typename Cplx<T>::type *spec, FFTPair &fft,
               double *part, cudaStream_t st);
// Adjoint of grf_device: dL/dw from dL/d(density) (dbar is overwritten).
template <typename T>
int grf_adjoint_device(const conan_ic_params &p, const Mesh &m, const T *w, T *dbar, T *wbar,
                       typename Cplx<T>::type *spec, typename Cplx<T>::type *spec2, T *tmp, FFTPair &fft,
                       double *part, cudaStream_t st);
// Density mesh -> potential mesh, in place (a symmetric operator: it is its
// own adjoint).
template <typename T>
int potential_device(const Mesh &m, double L, T *mesh, typename Cplx<T>::type *spec, FFTPair &fft,
                     cudaStream_t st);

}  // namespace conan
