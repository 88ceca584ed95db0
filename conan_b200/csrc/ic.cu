// ic.cu -- initial conditions on the GPU: white noise, the Gaussian random
// field of the `ic` tool (src/ic/ic.cc:37-98), its potential
// (src/ic/ic.cc:100-117) and the Zel'dovich displacement record
// (src/ic/ic.cc:119-146). Meshes are real with axis 0 fastest; all
// filtering happens on the R2C half spectrum.
#include <cmath>
#include <vector>

#include "fft.cuh"
#include "ic.cuh"
#include "pm.cuh"

namespace conan {

__global__ void k_noise_philox_f64(double *__restrict__ out, size_t n, unsigned long long seed) {
    size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * j >= n) return;
    double z0, z1;
    philox_normal_pair(seed, j, &z0, &z1);
    out[2 * j] = z0;
    if (2 * j + 1 < n) out[2 * j + 1] = z1;
}

template <typename T>
__global__ void k_noise_philox(T *__restrict__ out, size_t n, unsigned long long seed) {
    size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (2 * j >= n) return;
    double z0, z1;
    philox_normal_pair(seed, j, &z0, &z1);
    out[2 * j] = (T)z0;
    if (2 * j + 1 < n) out[2 * j + 1] = (T)z1;
}

// Filter value of half-spectrum element e (see ICFilter).
__device__ inline double ic_filter_value(const ICFilter &F, const Mesh &m, size_t e, bool with_s) {
    int kv[3];
    long long k2 = spec_k2(e, m, kv);
    if (F.mode == IC_CDM) {
        // CDM<R>, src/ic/ic.cc:14-35, at physical k (kspace(N, L)).
        double kk = sqrt((double)k2) * (2 * M_PI / F.L);
        const double e1 = 2.718281828459045, Theta = 2.7255 / 2.7, A = 1122670;
        double q = kk * Theta * Theta / (F.Omega0 * F.h), L0 = log(2 * e1 + 1.8 * q),
               C0 = 14.2 + 731.0 / (1 + 62.5 * q), T0 = L0 / (L0 + C0 * q * q);
        return sqrt(A * pow(kk, F.ns) * T0 * T0);
    }
    // Scale-free: k in radians per cell (kspace(N, N), src/ic/ic.cc:61-64),
    // sqrt(P(|k|)) with P = k^ns times Fourier::scale(t) (fourier.hh:79-100).
    double ks[3], s2 = 0;
    for (int a = 0; a < m.R; ++a) {
        ks[a] = kv[a] * (2 * M_PI / m.n);
        s2 += ks[a] * ks[a];
    }
    double p = sqrt(pow(sqrt(s2), F.ns));
    if (!with_s) return p;
    double s = 1.0;
    for (int a = 0; a < m.R; ++a) s *= exp(F.t * (cos(ks[a]) - 1));
    return p * s;
}

// Per-block sums of w |x_hat|^2 PS(k)^2 over the half spectrum (DC excluded):
// the variance of the smoothed field by Parseval.
template <typename T>
__global__ void k_ic_var(const typename Cplx<T>::type *__restrict__ spec, Mesh m, ICFilter F,
                         double *__restrict__ part) {
    double s = 0;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < m.spec;
         e += (size_t)gridDim.x * blockDim.x) {
        if (e == 0) continue;
        double f = ic_filter_value(F, m, e, true);
        auto z = spec[e];
        int kx = (int)(e % (size_t)m.nh);
        s += spec_weight(kx, m.n) * ((double)z.x * z.x + (double)z.y * z.y) * f * f;
    }
    s = block_sum<double>(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

template <typename T>
__global__ void k_ic_filter(typename Cplx<T>::type *__restrict__ spec, Mesh m, ICFilter F, bool with_s,
                            double scale) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.spec) return;
    double f = e == 0 ? 0.0 : ic_filter_value(F, m, e, with_s) * scale;
    auto z = spec[e];
    z.x = (T)((double)z.x * f);
    z.y = (T)((double)z.y * f);
    spec[e] = z;
}

// spec *= gsp / |n|^2 (physical -1/k^2 with the 1/size normalisation folded
// into gsp), DC = 0.
template <typename T>
__global__ void k_ic_potential(typename Cplx<T>::type *__restrict__ spec, Mesh m, double gsp) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.spec) return;
    int kv[3];
    long long k2 = spec_k2(e, m, kv);
    double g = k2 > 0 ? gsp / (double)k2 : 0.0;
    auto z = spec[e];
    z.x = (T)((double)z.x * g);
    z.y = (T)((double)z.y * g);
    spec[e] = z;
}

// out = in * i sin(2 pi n_axis / N) * scale (Fourier::derivative,
// src/base/fourier.hh:111-118, on kspace(N, N)).
template <typename T>
__global__ void k_ic_deriv(const typename Cplx<T>::type *__restrict__ in,
                           typename Cplx<T>::type *__restrict__ out, Mesh m, int axis, double scale) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.spec) return;
    int kv[3];
    spec_k2(e, m, kv);
    double s = sin(kv[axis] * (2 * M_PI / m.n)) * scale;
    auto z = in[e];
    typename Cplx<T>::type r;
    r.x = (T)(-(double)z.y * s);
    r.y = (T)((double)z.x * s);
    out[e] = r;
}

// AoS scatter of one component: out[i * R + c] = in[i].
template <typename T>
__global__ void k_interleave(const T *__restrict__ in, double *__restrict__ out, size_t n, int R, int c) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i * R + c] = (double)in[i];
}

int check_ic_params(const conan_ic_params *p) {
    if (!p) return set_error(CONAN_ERR_ARG, "null parameters");
    if (p->dim < 1 || p->dim > 3)
        return set_error(CONAN_ERR_UNSUPPORTED, "only 1, 2 and 3 dimensions supported (dim = %d)", p->dim);
    if (p->mbits < 1 || p->mbits > 12) return set_error(CONAN_ERR_ARG, "mbits = %d out of range", p->mbits);
    long long cells = 1;
    for (int i = 0; i < p->dim; ++i) cells *= 1LL << p->mbits;
    if (cells >= (1LL << 32)) return set_error(CONAN_ERR_ARG, "mesh of %lld cells too large", cells);
    if (!(p->size > 0)) return set_error(CONAN_ERR_ARG, "box size must be positive");
    if (p->precision != CONAN_FP32 && p->precision != CONAN_FP64)
        return set_error(CONAN_ERR_ARG, "precision must be CONAN_FP32 or CONAN_FP64");
    return CONAN_OK;
}

// Scoped device buffers and plan for one ic call.
template <typename T> struct ICWork {
    typedef typename Cplx<T>::type CT;
    Mesh m;
    T *mesh = nullptr;
    CT *spec = nullptr, *spec2 = nullptr;
    double *xfer = nullptr, *part = nullptr;
    void *work = nullptr;
    FFTPair fft;
    cudaStream_t st = nullptr;
    ~ICWork() {
        if (st) cudaStreamSynchronize(st);
        fft.destroy();
        cudaFree(mesh);
        cudaFree(spec);
        cudaFree(spec2);
        cudaFree(xfer);
        cudaFree(part);
        cudaFree(work);
        if (st) cudaStreamDestroy(st);
    }
    int setup(const conan_ic_params &p, bool need_spec2) {
        m = make_mesh(p.dim, 1 << p.mbits);
        CONAN_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CONAN_CUDA(cudaMalloc(&mesh, m.cells * sizeof(T)));
        CONAN_CUDA(cudaMalloc(&spec, m.spec * sizeof(CT)));
        if (need_spec2) CONAN_CUDA(cudaMalloc(&spec2, m.spec * sizeof(CT)));
        CONAN_CUDA(cudaMalloc(&xfer, m.cells * sizeof(double) * (need_spec2 ? p.dim : 1)));
        CONAN_CUDA(cudaMalloc(&part, 1024 * sizeof(double)));
        CONAN_TRY(fft.create(m, sizeof(T) == 8, 1));
        CONAN_CUDA(cudaMalloc(&work, fft.work_bytes ? fft.work_bytes : 16));
        CONAN_TRY(fft.bind(work, st));
        return CONAN_OK;
    }
    unsigned gc() const { return (unsigned)((m.cells + 255) / 256); }
    unsigned gs() const { return (unsigned)((m.spec + 255) / 256); }
    int upload(const double *h) {
        CONAN_CUDA(cudaMemcpyAsync(xfer, h, m.cells * sizeof(double), cudaMemcpyHostToDevice, st));
        k_convert<double, T><<<gc(), 256, 0, st>>>(xfer, mesh, m.cells, 1.0, 0.0);
        CONAN_LAUNCHED();
        return CONAN_OK;
    }
    int download(double *h) {
        k_convert<T, double><<<gc(), 256, 0, st>>>(mesh, xfer, m.cells, 1.0, 0.0);
        CONAN_LAUNCHED();
        CONAN_CUDA(cudaMemcpyAsync(h, xfer, m.cells * sizeof(double), cudaMemcpyDeviceToHost, st));
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }
};

// Device pipeline of _generate_random_field<R>, src/ic/ic.cc:37-98, on an
// already filled real mesh `mesh` (the noise); leaves the density in it.
template <typename T>
int grf_device(const conan_ic_params &p, const Mesh &m, T *mesh, typename Cplx<T>::type *spec, FFTPair &fft,
               double *part, cudaStream_t st) {
    CONAN_TRY(fft.forward(mesh, spec));
    ICFilter F{};
    F.ns = p.ns;
    F.L = p.size;
    F.Omega0 = p.Omega0;
    F.h = p.H0 / 100.0;
    unsigned gs = (unsigned)((m.spec + 255) / 256);
    if (p.scale_free) {
        F.mode = IC_SCALE_FREE;
        F.t = p.scale * m.n / p.size;  // Fourier::scale<R>(sigma * N/L), ic.cc:63
        const int nb = 512;
        k_ic_var<T><<<nb, 256, 0, st>>>(spec, m, F, part);
        CONAN_LAUNCHED();
        double h[nb];
        CONAN_CUDA(cudaMemcpyAsync(h, part, sizeof h, cudaMemcpyDeviceToHost, st));
        CONAN_CUDA(cudaStreamSynchronize(st));
        double acc = 0;
        for (int b = 0; b < nb; ++b) acc += h[b];
        double nc = (double)m.cells;
        double var = acc / (nc * nc);  // mean of the smoothed field squared
        double scale = p.sigma / (nc * std::sqrt(var));
        k_ic_filter<T><<<gs, 256, 0, st>>>(spec, m, F, p.smooth != 0, scale);
    } else {
        F.mode = IC_CDM;
        double res = p.size / m.n;
        double scale = 1.0 / ((double)m.cells * std::pow(res, 0.5 * m.R));
        k_ic_filter<T><<<gs, 256, 0, st>>>(spec, m, F, false, scale);
    }
    CONAN_LAUNCHED();
    CONAN_TRY(fft.inverse(spec, mesh));
    return CONAN_OK;
}
template int grf_device<float>(const conan_ic_params &, const Mesh &, float *, cufftComplex *, FFTPair &,
                               double *, cudaStream_t);
template int grf_device<double>(const conan_ic_params &, const Mesh &, double *, cufftDoubleComplex *,
                                FFTPair &, double *, cudaStream_t);

// _compute_potential<R>, src/ic/ic.cc:100-117, in place on a device mesh.
template <typename T>
int potential_device(const Mesh &m, double L, T *mesh, typename Cplx<T>::type *spec, FFTPair &fft,
                     cudaStream_t st) {
    CONAN_TRY(fft.forward(mesh, spec));
    double gsp = -std::pow(L / (2 * M_PI), 2) / (double)m.cells;
    k_ic_potential<T><<<(unsigned)((m.spec + 255) / 256), 256, 0, st>>>(spec, m, gsp);
    CONAN_LAUNCHED();
    CONAN_TRY(fft.inverse(spec, mesh));
    return CONAN_OK;
}
template int potential_device<float>(const Mesh &, double, float *, cufftComplex *, FFTPair &, cudaStream_t);
template int potential_device<double>(const Mesh &, double, double *, cufftDoubleComplex *, FFTPair &,
                                      cudaStream_t);

// out = in * f(k)^power * scale, DC = 0 (f the scale-free or CDM filter).
template <typename T>
__global__ void k_ic_filter_to(const typename Cplx<T>::type *__restrict__ in, typename Cplx<T>::type *__restrict__ out,
                               Mesh m, ICFilter F, bool with_s, int power, double scale) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.spec) return;
    double f = 0.0;
    if (e != 0) {
        double v = ic_filter_value(F, m, e, with_s);
        f = (power == 2 ? v * v : v) * scale;
    }
    auto z = in[e];
    typename Cplx<T>::type r;
    r.x = (T)((double)z.x * f);
    r.y = (T)((double)z.y * f);
    out[e] = r;
}

// Per-block sums of a . b (FP64, fixed order).
template <typename T>
__global__ void k_dot_partial(const T *__restrict__ a, const T *__restrict__ b, size_t n, double *__restrict__ part) {
    double s = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        s += (double)a[i] * (double)b[i];
    s = block_sum<double>(s);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// y += alpha x
template <typename T> __global__ void k_axpy(T *__restrict__ y, const T *__restrict__ x, size_t n, double alpha) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = (T)((double)y[i] + alpha * (double)x[i]);
}

static ICFilter filter_of(const conan_ic_params &p, const Mesh &m) {
    ICFilter F{};
    F.mode = p.scale_free ? IC_SCALE_FREE : IC_CDM;
    F.ns = p.ns;
    F.L = p.size;
    F.Omega0 = p.Omega0;
    F.h = p.H0 / 100.0;
    F.t = p.scale * m.n / p.size;
    return F;
}

template <typename T> static int host_sum(const double *part, int nb, cudaStream_t st, double *out) {
    std::vector<double> h(nb);
    CONAN_CUDA(cudaMemcpyAsync(h.data(), part, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    CONAN_CUDA(cudaStreamSynchronize(st));
    double acc = 0;
    for (int b = 0; b < nb; ++b) acc += h[b];
    *out = acc;
    return CONAN_OK;
}

// Adjoint of the Gaussian random field of grf_device: given the noise w and
// dL/d(density) in dbar (overwritten), writes dL/dw into wbar. Scale-free:
// density = s y with y = L_F w, s = sigma / sqrt(var), var = |L_PS w|^2 / N,
// L_X = C2R diag(X) R2C / N (DC = 0), all symmetric, so
//   wbar = s L_F dbar - (s / var) (y . dbar) / N  L_PS L_PS w.
// CDM: density = A w with A symmetric, wbar = A dbar.
// Scratch: spec, spec2 (half spectra), tmp (mesh); part >= 512 doubles.
template <typename T>
int grf_adjoint_device(const conan_ic_params &p, const Mesh &m, const T *w, T *dbar, T *wbar,
                       typename Cplx<T>::type *spec, typename Cplx<T>::type *spec2, T *tmp, FFTPair &fft,
                       double *part, cudaStream_t st) {
    const ICFilter F = filter_of(p, m);
    const unsigned gs = (unsigned)((m.spec + 255) / 256), gc = (unsigned)((m.cells + 255) / 256);
    const double nc = (double)m.cells;
    if (!p.scale_free) {
        double scale = 1.0 / (nc * std::pow(p.size / m.n, 0.5 * m.R));
        CONAN_TRY(fft.forward(dbar, spec));
        k_ic_filter_to<T><<<gs, 256, 0, st>>>(spec, spec, m, F, false, 1, scale);
        CONAN_LAUNCHED();
        CONAN_TRY(fft.inverse(spec, wbar));
        return CONAN_OK;
    }
    // W = R2C(w) (fft.forward leaves w intact for out-of-place R2C; copy to be safe)
    CONAN_CUDA(cudaMemcpyAsync(tmp, w, m.cells * sizeof(T), cudaMemcpyDeviceToDevice, st));
    CONAN_TRY(fft.forward(tmp, spec));
    const int nb = 512;
    k_ic_var<T><<<nb, 256, 0, st>>>(spec, m, F, part);
    CONAN_LAUNCHED();
    double acc;
    CONAN_TRY(host_sum<T>(part, nb, st, &acc));
    const double var = acc / (nc * nc), s = p.sigma / std::sqrt(var);
    // y = L_F w
    k_ic_filter_to<T><<<gs, 256, 0, st>>>(spec, spec2, m, F, p.smooth != 0, 1, 1.0 / nc);
    CONAN_LAUNCHED();
    CONAN_TRY(fft.inverse(spec2, tmp));
    k_dot_partial<T><<<nb, 256, 0, st>>>(tmp, dbar, m.cells, part);
    CONAN_LAUNCHED();
    double dot;
    CONAN_TRY(host_sum<T>(part, nb, st, &dot));
    // q = L_PS L_PS w into tmp
    k_ic_filter_to<T><<<gs, 256, 0, st>>>(spec, spec2, m, F, true, 2, 1.0 / nc);
    CONAN_LAUNCHED();
    CONAN_TRY(fft.inverse(spec2, tmp));
    // wbar = s L_F dbar
    CONAN_TRY(fft.forward(dbar, spec));
    k_ic_filter_to<T><<<gs, 256, 0, st>>>(spec, spec, m, F, p.smooth != 0, 1, s / nc);
    CONAN_LAUNCHED();
    CONAN_TRY(fft.inverse(spec, wbar));
    k_axpy<T><<<gc, 256, 0, st>>>(wbar, tmp, m.cells, -(s / var) * dot / nc);
    CONAN_LAUNCHED();
    return CONAN_OK;
}
template int grf_adjoint_device<float>(const conan_ic_params &, const Mesh &, const float *, float *, float *,
                                       cufftComplex *, cufftComplex *, float *, FFTPair &, double *, cudaStream_t);
template int grf_adjoint_device<double>(const conan_ic_params &, const Mesh &, const double *, double *,
                                        double *, cufftDoubleComplex *, cufftDoubleComplex *, double *, FFTPair &,
                                        double *, cudaStream_t);

template <typename T> int noise_device(const Mesh &m, unsigned long long seed, T *mesh, cudaStream_t st) {
    size_t pairs = (m.cells + 1) / 2;
    k_noise_philox<T><<<(unsigned)((pairs + 255) / 256), 256, 0, st>>>(mesh, m.cells, seed);
    CONAN_LAUNCHED();
    return CONAN_OK;
}
template int noise_device<float>(const Mesh &, unsigned long long, float *, cudaStream_t);
template int noise_device<double>(const Mesh &, unsigned long long, double *, cudaStream_t);

template <typename T> int ic_generate(const conan_ic_params &p, const double *noise, double *out) {
    ICWork<T> w;
    CONAN_TRY(w.setup(p, false));
    if (noise)
        CONAN_TRY(w.upload(noise));
    else
        CONAN_TRY(noise_device<T>(w.m, p.seed, w.mesh, w.st));
    CONAN_TRY(grf_device<T>(p, w.m, w.mesh, w.spec, w.fft, w.part, w.st));
    return w.download(out);
}

template <typename T> int ic_potential(const conan_ic_params &p, double *inout) {
    ICWork<T> w;
    CONAN_TRY(w.setup(p, false));
    CONAN_TRY(w.upload(inout));
    CONAN_TRY(potential_device<T>(w.m, p.size, w.mesh, w.spec, w.fft, w.st));
    return w.download(inout);
}

template <typename T> int ic_displacement(const conan_ic_params &p, const double *pot, double *psi) {
    ICWork<T> w;
    CONAN_TRY(w.setup(p, true));
    CONAN_TRY(w.upload(pot));
    CONAN_TRY(w.fft.forward(w.mesh, w.spec));
    double scale = 1.0 / ((double)w.m.cells / p.size * w.m.n);  // real_part(size / L * N)
    for (int a = 0; a < p.dim; ++a) {
        k_ic_deriv<T><<<w.gs(), 256, 0, w.st>>>(w.spec, w.spec2, w.m, a, scale);
        CONAN_LAUNCHED();
        CONAN_TRY(w.fft.inverse(w.spec2, w.mesh));
        k_interleave<T><<<w.gc(), 256, 0, w.st>>>(w.mesh, w.xfer, w.m.cells, p.dim, a);
        CONAN_LAUNCHED();
    }
    CONAN_CUDA(cudaMemcpyAsync(psi, w.xfer, w.m.cells * p.dim * sizeof(double), cudaMemcpyDeviceToHost, w.st));
    CONAN_CUDA(cudaStreamSynchronize(w.st));
    return CONAN_OK;
}

}  // namespace conan

using namespace conan;

extern "C" {

int conan_ic_noise(const conan_ic_params *p, double *noise_out) {
    CONAN_TRY(check_ic_params(p));
    if (!noise_out) return set_error(CONAN_ERR_ARG, "null output");
    CONAN_TRY(device_guard(p->device));
    ICWork<double> w;
    CONAN_TRY(w.setup(*p, false));
    size_t pairs = (w.m.cells + 1) / 2;
    k_noise_philox_f64<<<(unsigned)((pairs + 255) / 256), 256, 0, w.st>>>(w.xfer, w.m.cells, p->seed);
    CONAN_LAUNCHED();
    CONAN_CUDA(cudaMemcpyAsync(noise_out, w.xfer, w.m.cells * sizeof(double), cudaMemcpyDeviceToHost, w.st));
    CONAN_CUDA(cudaStreamSynchronize(w.st));
    return CONAN_OK;
}

int conan_ic_generate(const conan_ic_params *p, const double *noise_or_null, double *density_out) {
    CONAN_TRY(check_ic_params(p));
    if (!density_out) return set_error(CONAN_ERR_ARG, "null output");
    CONAN_TRY(device_guard(p->device));
    return p->precision == CONAN_FP64 ? ic_generate<double>(*p, noise_or_null, density_out)
                                      : ic_generate<float>(*p, noise_or_null, density_out);
}

int conan_ic_potential(const conan_ic_params *p, double *inout) {
    CONAN_TRY(check_ic_params(p));
    if (!inout) return set_error(CONAN_ERR_ARG, "null buffer");
    CONAN_TRY(device_guard(p->device));
    return p->precision == CONAN_FP64 ? ic_potential<double>(*p, inout) : ic_potential<float>(*p, inout);
}

int conan_ic_displacement(const conan_ic_params *p, const double *potential, double *psi_out) {
    CONAN_TRY(check_ic_params(p));
    if (!potential || !psi_out) return set_error(CONAN_ERR_ARG, "null buffer");
    CONAN_TRY(device_guard(p->device));
    return p->precision == CONAN_FP64 ? ic_displacement<double>(*p, potential, psi_out)
                                      : ic_displacement<float>(*p, potential, psi_out);
}

}  // extern "C"
