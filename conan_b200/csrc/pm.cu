// pm.cu -- the particle-mesh solver handle (conan_pm_*), the B200
// replacement of the reference's Gravity<R> solver (src/run/nbody.hh:53-219)
// driven by LeapFrog::run (src/run/leapfrog.hh:33-46).
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "fft.cuh"
#include "fft_plane.cuh"
// The forward plane pass zeroes the accumulator behind its reads (1) or a
// memset does it afterwards (0); a compile-time tunable.
#ifndef PLANE_CLEAR
#define PLANE_CLEAR 1
#endif
#include "fft_z.cuh"
#include "ic.cuh"
#include "pm.cuh"

#include <type_traits>

namespace conan {

std::string &last_error() {
    static thread_local std::string s;
    return s;
}

int set_error(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    last_error() = buf;
    return code;
}

int err_word_status(int h) {
    if (!h) return CONAN_OK;
    if (h & 8)
        return set_error(CONAN_ERR_TIMEOUT,
                         "a bounded wait for a bulk tensor copy into shared memory ran out (code %d)", h);
    return set_error(CONAN_ERR_STATE, "kernel self-check failed (code %d): corrupt cell offsets or payload", h);
}

double adot(double H0, double Om, double OL, double a) {
    // Cosmology::operator(), src/run/cosmology.hh:16-23.
    double Ok = 1 - Om - OL;
    return H0 * a * std::sqrt(OL + Om * std::pow(a, -3) + Ok * std::pow(a, -2));
}

int check_pm_params(const conan_pm_params *p) {
    if (!p) return set_error(CONAN_ERR_ARG, "null parameters");
    if (p->dim < 1 || p->dim > 3)
        return set_error(CONAN_ERR_UNSUPPORTED, "dim = %d: the GPU path supports 1, 2 and 3 dimensions",
                         p->dim);
    if (!is_pow2(p->n_mass) || p->n_mass < 2)
        return set_error(CONAN_ERR_ARG, "n_mass = %d must be a power of two >= 2", p->n_mass);
    if (!is_pow2(p->f)) return set_error(CONAN_ERR_ARG, "f = %d must be a power of two >= 1", p->f);
    long long nf = (long long)p->n_mass * p->f;
    long long cells = 1;
    for (int i = 0; i < p->dim; ++i) cells *= nf;
    if (cells >= (1LL << 32))
        return set_error(CONAN_ERR_ARG, "force mesh of %lld cells exceeds 2^32 - 1", cells);
    if (!(p->size > 0)) return set_error(CONAN_ERR_ARG, "box size must be positive");
    if (p->precision != CONAN_FP32 && p->precision != CONAN_FP64)
        return set_error(CONAN_ERR_ARG, "precision must be CONAN_FP32 or CONAN_FP64");
    if (p->gradient != CONAN_GRAD_FD4 && p->gradient != CONAN_GRAD_SPECTRAL)
        return set_error(CONAN_ERR_ARG, "gradient must be CONAN_GRAD_FD4 or CONAN_GRAD_SPECTRAL");
    if (!(p->H0 > 0)) return set_error(CONAN_ERR_ARG, "H0 must be positive");
    return CONAN_OK;
}

int device_guard(int dev) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
        return set_error(CONAN_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    if (dev < 0 || dev >= n) return set_error(CONAN_ERR_ARG, "device %d out of range (%d devices)", dev, n);
    CONAN_CUDA(cudaSetDevice(dev));
    return CONAN_OK;
}

// ------------------------------------------------------------------ PM --

template <typename T, int R> struct PM : PMBase {
    typedef typename Cplx<T>::type CT;
    typedef typename Pay<T>::elem PE;

    conan_pm_params prm{};
    Mesh mf{}, mm{};
    size_t np = 0;
    double res_f = 0, res_m = 0, mass = 1, G = 0;
    Parts<T> P{};
    T *mesh = nullptr;
    T *gm[3] = {nullptr, nullptr, nullptr};
    G4<T> *grad = nullptr;  // packed FD4 gradient mesh
    CT *spec = nullptr, *spec2 = nullptr;
    uint32_t *count = nullptr, *off = nullptr, *rank = nullptr, *bsum = nullptr;
    int *err = nullptr;  // device error word set by kernel self-checks
    PE *pay = nullptr;
    // Host transfers pass through two staging chunks of stage_n doubles each,
    // allocated at creation: no transfer allocates device memory, and the
    // chunks alternate on the handle's stream.
    double *stage[2] = {nullptr, nullptr};
    size_t stage_n = 0;
    static constexpr size_t STAGE_MAX = (size_t)1 << 24;  // doubles per chunk (128 MiB)
    void *work = nullptr;
    FFTPair fft;
    // FP32 3D FD4 meshes of 64..1024 cells per side: the Poisson solve as 2D
    // transforms of the z planes around the shared-memory z pass (fft_z.cuh)
    FFTPair fft2;
    float2 *ztw = nullptr;  // exp(-2 pi i k / n), k < n
    bool zpass = false;
    cudaStream_t st = nullptr;
    Profiler prof;
    std::vector<void *> allocs;
    double a_pos = 0, a_mom = 0;
    bool ranks_pending = false;
    int mesh_holds = 0;  // 0 nothing, 1 delta, 2 phi
    unsigned cb_every = 1;
    size_t bytes = 0;

    ~PM() override {
        if (st) cudaStreamSynchronize(st);
        if (gexec) cudaGraphExecDestroy(gexec);
        fft.destroy();
        fft2.destroy();
        for (void *p : allocs) cudaFree(p);
        if (st) cudaStreamDestroy(st);
    }

    template <typename U> int alloc(U **p, size_t n) {
        void *q = nullptr;
        size_t b = n * sizeof(U);
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&q, b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return set_error(CONAN_ERR_ALLOC, "cudaMalloc of %zu bytes failed: %s", b, cudaGetErrorString(e));
        }
        allocs.push_back(q);
        bytes += b;
        *p = (U *)q;
        return CONAN_OK;
    }

    // `batch` equal boxes stored back to back (ensembles); 1 for conan_pm.
    int create(const conan_pm_params &p, int batch = 1) {
        prm = p;
        int nf = p.n_mass * p.f;
        mf = make_mesh(R, nf, batch);
        mm = make_mesh(R, p.n_mass, batch);
        np = mm.cells;
        res_f = p.size / nf;
        res_m = p.size / p.n_mass;
        mass = std::pow(double(nf) / p.n_mass, R);  // src/run/nbody.hh:85
        G = 3. / 2 * p.Omega_m * p.H0 * p.H0;       // src/run/cosmology.hh:13
        CONAN_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        P.np = np;
        P.mshift = mm.shift;
        P.f = p.f;
        P.bshift = R * mm.shift;
        for (int k = 0; k < R; ++k) {
            CONAN_TRY(alloc(&P.d[k], np));
            CONAN_TRY(alloc(&P.p[k], np));
        }
        CONAN_TRY(alloc(&mesh, mf.cells));
        CONAN_TRY(alloc(&spec, mf.spec));
        if (p.gradient == CONAN_GRAD_SPECTRAL) {
            CONAN_TRY(alloc(&spec2, mf.spec));
            for (int k = 0; k < R; ++k) CONAN_TRY(alloc(&gm[k], mf.cells));
        } else {
            CONAN_TRY(alloc(&grad, mf.cells));
        }
        CONAN_TRY(alloc(&count, mf.cells));
        CONAN_TRY(alloc(&off, mf.cells + 1));
        CONAN_TRY(alloc(&rank, np));
        size_t nb = (mf.cells + SCAN_CHUNK - 1) / SCAN_CHUNK;
        CONAN_TRY(alloc(&bsum, nb));
        CONAN_TRY(alloc(&pay, np * Pay<T>::words));
        stage_n = std::min(STAGE_MAX, std::max(np * (size_t)R, std::max(mf.cells, mm.cells)));
        CONAN_TRY(alloc(&stage[0], stage_n));
        CONAN_TRY(alloc(&stage[1], stage_n));
        CONAN_TRY(alloc(&err, 1));
        CONAN_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        CONAN_CUDA(cudaMemsetAsync(count, 0, mf.cells * sizeof(uint32_t), st));
        bool lag = sizeof(T) == 4 && (lag_try<0>() || lag_try<1>() || lag_try<2>());
        // On fine meshes (f >= 2) a window that fits shared memory only fits
        // a small tile and holds many cells per particle, each of which gets
        // about one corner: clearing and flushing it costs more than the
        // atomics it saves. Deposit directly from the largest tile then.
        if (sizeof(T) == 4 && (!lag || (double)lwin.cells > LAG_WINDOW_CELLS_PER_PARTICLE * lag_particles()))
            lag = lag_try<0>(true) || lag_try<1>(true) || lag_try<2>(true);
        if (lag) {
            CONAN_TRY(alloc(&lacc, mf.cells));
            CONAN_CUDA(cudaMemsetAsync(lacc, 0, mf.cells * sizeof(unsigned long long), st));
            dep_variant = DEP_LAG;
            CONAN_TRY(tma_setup());
            pers = LAG_PERSIST != 0;
            CONAN_TRY(pers_setup());
        }
        CONAN_TRY(fft.create(mf, sizeof(T) == 8, batch));
        size_t wbytes = fft.work_bytes;
        if (sizeof(T) == 4 && R == 3 && p.gradient == CONAN_GRAD_FD4 && mf.n >= 64 && mf.n <= 1024) {
            CONAN_TRY(fft2.create_planes(mf, false, batch));
            CONAN_TRY(zpass_setup());
            wbytes = std::max(wbytes, fft2.work_bytes);
            zpass = true;
            if (lacc) CONAN_TRY(plane_setup());
        }
        // CONAN_GRAD_KERNEL: cell or zm picks the gradient-mesh kernel at
        // creation (before any autotuning)
        if (const char *gk = getenv("CONAN_GRAD_KERNEL")) grad_zm = !strcmp(gk, "zm");
        CONAN_TRY(alloc((char **)&work, wbytes));
        CONAN_TRY(fft.bind(work, st));
        if (zpass) CONAN_TRY(fft2.bind(work, st));
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }

    // Particles per staging chunk (whole particles of R doubles).
    size_t stage_particles() const { return stage_n / (size_t)R; }

    // Absolute FP64 state of the n particles of view v into host X, Pm
    // (either may be null), chunk by chunk through the staging buffers;
    // returns after the last copy.
    int export_state(const Parts<T> &v, size_t n, double *X, double *Pm) {
        const size_t cp = stage_particles();
        for (size_t i0 = 0; i0 < n; i0 += cp) {
            const size_t cnt = std::min(cp, n - i0);
            CONAN_TIMED(prof, "export", st,
                        (k_export<T, R><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(
                            v, res_f, i0, cnt, X ? stage[0] : nullptr, Pm ? stage[1] : nullptr)));
            if (X)
                CONAN_CUDA(cudaMemcpyAsync(X + i0 * R, stage[0], cnt * R * sizeof(double), cudaMemcpyDeviceToHost,
                                           st));
            if (Pm)
                CONAN_CUDA(cudaMemcpyAsync(Pm + i0 * R, stage[1], cnt * R * sizeof(double), cudaMemcpyDeviceToHost,
                                           st));
        }
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }

    // Converts n host doubles into the device array out (type T), chunk by
    // chunk through the staging buffers.
    int upload_mesh(const double *in, T *out, size_t n) {
        for (size_t c0 = 0, b = 0; c0 < n; c0 += stage_n, b ^= 1) {
            const size_t cnt = std::min(stage_n, n - c0);
            CONAN_CUDA(cudaMemcpyAsync(stage[b], in + c0, cnt * sizeof(double), cudaMemcpyHostToDevice, st));
            CONAN_TIMED(prof, "convert", st,
                        (k_convert<double, T><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(stage[b], out + c0, cnt,
                                                                                          1.0, 0.0)));
        }
        return CONAN_OK;
    }

    dim3 grid_p() const { return dim3((unsigned)((np + 255) / 256)); }

    // --- deposit ---------------------------------------------------------
    // 0 .. DEP_VARIANTS-1: sorted deposit with tile shape DepTile<R, V>;
    // DEP_LAG: Lagrangian-window deposit (FP32). Chosen by the autotuner.
    static constexpr int DEP_LAG = DEP_VARIANTS;
    int dep_variant = 0;

    // Lagrangian deposit: accumulator mesh, lattice-tile variant and window.
    unsigned long long *lacc = nullptr;
    int lag_v = -1;  // LagTile<R, V> variant that fits this mesh, -1: none
    LagWin lwin{};
    size_t lag_smem = 0;

    bool lag_on() const { return sizeof(T) == 4 && dep_variant == DEP_LAG && lag_v >= 0 && lacc; }

    template <int V> static constexpr double lag_tile_particles() {
        return (double)LagTile<R, V>::LX * LagTile<R, V>::LY * LagTile<R, V>::LZ;
    }
    double lag_particles() const {
        return lag_v == 0 ? lag_tile_particles<0>() : lag_v == 1 ? lag_tile_particles<1>() : lag_tile_particles<2>();
    }

    // direct: a window of two cells per axis, so that (nearly) every corner
    // goes straight to the accumulator mesh with one integer atomic.
    template <int V> bool lag_try(bool direct = false) {
        typedef LagTile<R, V> L;
        const int n = mm.n;
        if (n < L::LX || (R >= 2 && n < L::LY) || (R == 3 && n < L::LZ)) return false;
        LagWin w{};
        w.w[0] = direct ? 2 : L::LX * prm.f + L::M;
        w.w[1] = R >= 2 ? (direct ? 2 : L::LY * prm.f + L::M) : 1;
        w.w[2] = R == 3 ? (direct ? 2 : L::LZ * prm.f + L::M) : 1;
        w.cells = (w.w[0] * w.w[1] * w.w[2] + 3) & ~3;
        size_t sh = (size_t)w.cells * LAG_PLANES * sizeof(uint32_t);
        if (sh > 112 * 1024) return false;
        if constexpr (sizeof(T) == 4) {  // set once here, outside any stream capture
            auto kern = k_deposit_lag<R, L::LX, L::LY, L::LZ, L::THREADS>;
            auto fused = k_gkd_lag<R, L::LX, L::LY, L::LZ, L::THREADS>;
            if (!raise_dyn_smem(kern, sh) || !raise_dyn_smem(fused, sh)) return false;
        }
        lwin = w;
        lag_smem = sh;
        lag_v = V;
        return true;
    }

    template <int V> int launch_lag() {
        if constexpr (sizeof(T) == 4) {
            typedef LagTile<R, V> L;
            size_t tiles = (size_t)(mm.n / L::LX) * (R >= 2 ? mm.n / L::LY : 1) * (R == 3 ? mm.n / L::LZ : 1) *
                           (size_t)mm.batch;
            auto kern = k_deposit_lag<R, L::LX, L::LY, L::LZ, L::THREADS>;
            CONAN_TIMED(prof, "deposit", st, (kern<<<(unsigned)tiles, L::THREADS, lag_smem, st>>>(P, mf, lwin, lacc)));
            return CONAN_OK;
        } else {
            return set_error(CONAN_ERR_UNSUPPORTED, "the Lagrangian deposit is FP32 only");
        }
    }

    // The fused gather/kick/drift + deposit of variant V (FP32, FD4).
    // TMA staging of the 3D tile's particle arrays (FP32, 32x8x8 tiles):
    // tensor maps over d[k], p[k] built once at creation.
    TileMaps tmaps{};
    bool tma_ok = false;
    size_t tma_smem = 0;

    int tma_setup() {
        tma_ok = false;
        if constexpr (sizeof(T) == 4 && R == 3) {
            const char *off = getenv("CONAN_NO_TMA");
            if (off && *off && *off != '0') return CONAN_OK;
            if (lag_v == 0) return tma_setup_v<0>();
            if (lag_v == 1) return tma_setup_v<1>();
            if (lag_v == 2) return tma_setup_v<2>();
        }
        return CONAN_OK;
    }

    // Tensor maps over d[k], p[k] with the box of one particle group of
    // lattice tile V (LX x LY x THREADS / (LX LY)), and the staged kernel's
    // shared memory; tma_ok stays false when anything is missing (the
    // kernels then read global memory directly).
    template <int V> int tma_setup_v() {
        typedef LagTile<3, V> L;
        typedef CUresult (*Encode)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn) {
            cudaGetLastError();
            return CONAN_OK;
        }
        const cuuint64_t n = (cuuint64_t)mm.n;
        const cuuint64_t dims[3] = {n, n, n * (cuuint64_t)mm.batch};
        const cuuint64_t strides[2] = {n * 4, n * n * 4};
        // one z-plane of the tile per copy
        const cuuint32_t box[3] = {L::LX, L::LY, 1}, estr[3] = {1, 1, 1};
        float *arr[6] = {P.d[0], P.d[1], P.d[2], P.p[0], P.p[1], P.p[2]};
        for (int a = 0; a < 6; ++a)
            if (((Encode)fn)(&tmaps.a[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, arr[a], dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return CONAN_OK;
        const size_t stage_bytes = (size_t)(6 * L::LX * L::LY * L::LZ * 4 + 128);
        // the window after the staged arrays, or over them
        tma_smem = LAG_STAGE_KEEP ? stage_bytes + lag_smem : std::max(lag_smem, stage_bytes);
        auto kern = k_gkd_lag_tma<3, L::LX, L::LY, L::LZ, L::THREADS>;
        if (!raise_dyn_smem(kern, tma_smem)) return CONAN_OK;
        tma_ok = true;
        return CONAN_OK;
    }

    // Persistent staged launch (3D, lattice tiles 32x8x8 and 16x8x8 with twice
    // the threads, two staging buffers): on when `pers` and its set-up
    // succeeded for the current tile variant.
    bool pers = false, pers_ok = false;
    unsigned pers_grid = 0;
    size_t pers_smem = 0;
    template <int V> struct PersT {
        typedef LagTile<3, V> L;
        static constexpr int THREADS = 2 * L::THREADS;
    };
    int pers_setup() {
        pers_ok = false;
        if constexpr (sizeof(T) == 4 && R == 3) {
            if (!pers || !tma_ok || lag_v > 1) return CONAN_OK;
            return lag_v == 0 ? pers_setup_v<0>() : pers_setup_v<1>();
        }
        return CONAN_OK;
    }
    template <int V> int pers_setup_v() {
        typedef LagTile<3, V> L;
        constexpr int TH = PersT<V>::THREADS;
        auto kern = k_gkd_lag_pers<3, L::LX, L::LY, L::LZ, TH>;
        pers_smem = 128 + 2 * 6 * (size_t)(L::LX * L::LY * L::LZ) * 4 + lag_smem;
        if (!raise_dyn_smem(kern, pers_smem)) return CONAN_OK;
        int nb = 0, sms = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, TH, pers_smem) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, prm.device) != cudaSuccess || nb < 1) {
            cudaGetLastError();
            return CONAN_OK;
        }
        pers_grid = (unsigned)(nb * sms);
        pers_ok = true;
        return CONAN_OK;
    }

    template <int V> int launch_gkd_lag(const GKD &c, const char *name) {
        if constexpr (sizeof(T) == 4) {
            typedef LagTile<R, V> L;
            size_t tiles = (size_t)(mm.n / L::LX) * (R >= 2 ? mm.n / L::LY : 1) * (R == 3 ? mm.n / L::LZ : 1) *
                           (size_t)mm.batch;
            if constexpr (R == 3 && V <= 1) {
                if (pers_ok && tma_ok && (LAG_TMA_GATHER || !c.kick)) {
                    constexpr int TH = PersT<V>::THREADS;
                    auto pk = k_gkd_lag_pers<3, L::LX, L::LY, L::LZ, TH>;
                    const unsigned grid = (unsigned)std::min<size_t>(pers_grid, tiles);
                    CONAN_TIMED(prof, name, st,
                                (pk<<<grid, TH, pers_smem, st>>>(P, mf, grad, c, lwin, lacc, tmaps, err,
                                                                  (unsigned)tiles)));
                    return CONAN_OK;
                }
            }
            if constexpr (R == 3) {
                // staged (512^3, 32x8x8 tiles): drift+deposit 1.87 against 2.33
                // ms; with the gather, keeping the drifted displacements in the
                // staged memory and a one-plane window 3.55 against 3.76 ms
                if (tma_ok && (LAG_TMA_GATHER || !c.kick)) {
                    auto tk = k_gkd_lag_tma<3, L::LX, L::LY, L::LZ, L::THREADS>;
                    const int rec = prof.begin(name, st);
                    tk<<<(unsigned)tiles, L::THREADS, tma_smem, st>>>(P, mf, grad, c, lwin, lacc, tmaps, err);
                    cudaError_t e = cudaGetLastError();
                    if (e != cudaSuccess)
                        return set_error(CONAN_ERR_CUDA,
                                         "staged launch failed: %s (tile %dx%dx%d, %d threads, %zu tiles, %zu bytes "
                                         "shared, window %d cells)",
                                         cudaGetErrorString(e), L::LX, L::LY, L::LZ, L::THREADS, tiles, tma_smem,
                                         lwin.cells);
                    prof.end(rec, st);
                    return CONAN_OK;
                }
            }
            auto kern = k_gkd_lag<R, L::LX, L::LY, L::LZ, L::THREADS>;
            CONAN_TIMED(prof, name, st,
                        (kern<<<(unsigned)tiles, L::THREADS, lag_smem, st>>>(P, mf, grad, c, lwin, lacc)));
            return CONAN_OK;
        } else {
            return set_error(CONAN_ERR_UNSUPPORTED, "the Lagrangian deposit is FP32 only");
        }
    }

    // lag_ready: the accumulator holds the deposit of the current positions,
    // made by the fused kernel and not yet turned into the density mesh.
    bool lag_ready = false;
    int drop_lag_deposit() {
        if (lag_ready) CONAN_CUDA(cudaMemsetAsync(lacc, 0, mf.cells * sizeof(unsigned long long), st));
        lag_ready = false;
        return CONAN_OK;
    }

    // Particle positions were replaced: ranks and a fused deposit are stale.
    int positions_reset() {
        if (ranks_pending) CONAN_CUDA(cudaMemsetAsync(count, 0, mf.cells * sizeof(uint32_t), st));
        ranks_pending = false;
        return drop_lag_deposit();
    }

    // The Lagrangian deposit of the current positions into the accumulator
    // mesh (unless the fused gather kernel did it already).
    int lag_accumulate() {
        if (!lag_ready) {
            if (lag_v == 0) CONAN_TRY(launch_lag<0>());
            else if (lag_v == 1) CONAN_TRY(launch_lag<1>());
            else CONAN_TRY(launch_lag<2>());
        }
        lag_ready = false;
        return CONAN_OK;
    }

    int deposit_lag() {
        CONAN_TRY(lag_accumulate());
        size_t nt = (mf.cells + 3) / 4;  // four cells per thread
        CONAN_TIMED(prof, "deposit_mesh", st,
                    (k_acc_mesh<T><<<(unsigned)((nt + 255) / 256), 256, 0, st>>>(lacc, mesh, mf.cells, mass)));
        CONAN_TIMED(prof, "deposit_clear", st,
                    CONAN_CUDA(cudaMemsetAsync(lacc, 0, mf.cells * sizeof(unsigned long long), st)));
        mesh_holds = 1;
        return CONAN_OK;
    }

    // CONAN_DEPOSIT_SORTED or CONAN_DEPOSIT_LAGRANGIAN.
    int set_deposit(int mode) override {
        CONAN_TRY(drop_lag_deposit());  // a pending fused deposit belongs to the old mode
        if (mode == CONAN_DEPOSIT_SORTED) {
            dep_variant = 0;
            return CONAN_OK;
        }
        if (mode == CONAN_DEPOSIT_LAGRANGIAN) {
            if (sizeof(T) != 4 || lag_v < 0 || !lacc)
                return set_error(CONAN_ERR_UNSUPPORTED,
                                 "the Lagrangian deposit needs FP32 and a lattice of at least one tile per axis");
            dep_variant = DEP_LAG;
            return CONAN_OK;
        }
        return set_error(CONAN_ERR_ARG, "unknown deposit mode %d", mode);
    }
    int get_deposit(int *mode) override {
        if (!mode) return set_error(CONAN_ERR_ARG, "null mode");
        *mode = lag_on() ? CONAN_DEPOSIT_LAGRANGIAN : CONAN_DEPOSIT_SORTED;
        return CONAN_OK;
    }

    // Tiled deposit with tile variant V; returns 1 when V does not fit the
    // mesh (the caller falls back), CONAN_OK or an error code.
    template <int V> int deposit_tiles(double scale) {
        typedef DepTile<R, V> D;
        if (mf.n < D::TX || mf.n < D::TY || mf.n < D::TZ) return 1;
        size_t tiles = (size_t)(mf.n / D::TX) * (R >= 2 ? mf.n / D::TY : 1) * (R == 3 ? mf.n / D::TZ : 1) *
                       (size_t)mf.batch;
        constexpr size_t sh = deposit_smem<T, R, V>();
        auto kern = k_deposit<T, R, D::TX, D::TY, D::TZ, D::THREADS>;
        if (sh > 48 * 1024)
            CONAN_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
        CONAN_TIMED(prof, "deposit", st,
                    (kern<<<(unsigned)tiles, D::THREADS, sh, st>>>(off, pay, mesh, mf, scale, (uint32_t)np, err)));
        return CONAN_OK;
    }

    int rank_pass() {
        if (ranks_pending) CONAN_CUDA(cudaMemsetAsync(count, 0, mf.cells * sizeof(uint32_t), st));
        CONAN_TIMED(prof, "rank", st, (k_rank<T, R><<<grid_p(), 256, 0, st>>>(P, mf, count, rank)));
        ranks_pending = true;
        return CONAN_OK;
    }

    int deposit() {
        if (lag_on()) return deposit_lag();
        if (!ranks_pending) CONAN_TRY(rank_pass());
        size_t nb = (mf.cells + SCAN_CHUNK - 1) / SCAN_CHUNK;
        CONAN_TIMED(prof, "scan", st,
                    (k_scan_partial<<<(unsigned)nb, SCAN_T, 0, st>>>(count, mf.cells, bsum)));
        CONAN_TIMED(prof, "scan", st, (k_scan_blocks<<<1, 1024, 0, st>>>(bsum, (int)nb)));
        CONAN_TIMED(prof, "scan", st,
                    (k_scan_final<<<(unsigned)nb, SCAN_T, 0, st>>>(count, mf.cells, bsum, off)));
        ranks_pending = false;
        CONAN_TIMED(prof, "scatter", st,
                    (k_scatter<T, R><<<grid_p(), 256, 0, st>>>(P, mf, off, rank, pay, nullptr)));
        double scale = mass;
        int rc = 1;  // 1: the variant does not fit this mesh
        if (dep_variant == 1) rc = deposit_tiles<1>(scale);
        if (dep_variant == 2) rc = deposit_tiles<2>(scale);
        if (rc == 1) rc = deposit_tiles<0>(scale);
        if (rc > 1) return rc;
        if (rc == 1) {
            CONAN_TIMED(prof, "deposit", st,
                        (k_deposit_pull<T, R><<<(unsigned)((mf.cells + 255) / 256), 256, 0, st>>>(
                            off, pay, mesh, mf, scale)));
        }
        mesh_holds = 1;
        return CONAN_OK;
    }

    // --- Poisson: mesh (delta) -> mesh (phi) [and gradient meshes] ------
    // Green's function multiply of the half spectrum s (one CTA per row).
    int green(CT *s, double gs) {
        const unsigned rows = (unsigned)(mf.spec / (size_t)mf.nh);
        const int threads = mf.nh >= 256 ? 256 : ((mf.nh + 31) / 32) * 32;
        CONAN_TIMED(prof, "green", st, (k_green<T><<<rows, threads, 0, st>>>(s, mf, (T)gs)));
        return CONAN_OK;
    }

    int zpass_setup() {
        std::vector<float2> w((size_t)mf.n);
        for (int k = 0; k < mf.n; ++k) {
            const double a = -2.0 * M_PI * (double)k / (double)mf.n;
            w[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        CONAN_TRY(alloc(&ztw, (size_t)mf.n));
        CONAN_CUDA(cudaMemcpy(ztw, w.data(), w.size() * sizeof(float2), cudaMemcpyHostToDevice));
        switch (mf.n) {
            case 64: return zpass_attr<64>();
            case 128: return zpass_attr<128>();
            case 256: return zpass_attr<256>();
            case 512: return zpass_attr<512>();
            default: return zpass_attr<1024>();
        }
    }
    // z-pass lines per CTA: 0 the default width, else TX (the autotuner's knob)
    int ztx = 0;
    template <int N, int TX> int zpass_attr1() {
        if constexpr (ZTile<N, TX>::OK)
            if (!raise_dyn_smem(k_zpass_green<N, TX>, ZTile<N, TX>::SMEM))
                return set_error(CONAN_ERR_CUDA, "z pass: %zu bytes of shared memory refused", ZTile<N, TX>::SMEM);
        return CONAN_OK;
    }
    template <int N> int zpass_attr() {
        constexpr int T0 = ZTile<N>::TX;
        CONAN_TRY((zpass_attr1<N, 0>()));
        CONAN_TRY((zpass_attr1<N, T0 / 2>()));
        return zpass_attr1<N, 2 * T0>();
    }
    // widths of the z pass at this mesh size (default first)
    std::vector<int> zpass_widths() const {
        std::vector<int> w{0};
        auto add = [&](auto tag) {
            constexpr int N = decltype(tag)::value;
            constexpr int T0 = ZTile<N>::TX;
            if (ZTile<N, T0 / 2>::OK) w.push_back(T0 / 2);
            if (ZTile<N, 2 * T0>::OK) w.push_back(2 * T0);
        };
        switch (mf.n) {
            case 64: add(std::integral_constant<int, 64>()); break;
            case 128: add(std::integral_constant<int, 128>()); break;
            case 256: add(std::integral_constant<int, 256>()); break;
            case 512: add(std::integral_constant<int, 512>()); break;
            default: add(std::integral_constant<int, 1024>()); break;
        }
        return w;
    }
    template <int N, int TX> void zpass_launch1(float gs) {
        if constexpr (ZTile<N, TX>::OK) {
            typedef ZTile<N, TX> Z;
            const dim3 grid((unsigned)((mf.nh + Z::TX - 1) / Z::TX), (unsigned)mf.n, (unsigned)mf.batch);
            k_zpass_green<N, TX><<<grid, Z::THREADS, Z::SMEM, st>>>(reinterpret_cast<float2 *>(spec), mf, gs, ztw);
        }
    }
    template <int N> void zpass_launch(float gs) {
        constexpr int T0 = ZTile<N>::TX;
        if (ztx == T0 / 2 && ZTile<N, T0 / 2>::OK) zpass_launch1<N, T0 / 2>(gs);
        else if (ztx == 2 * T0 && ZTile<N, 2 * T0>::OK) zpass_launch1<N, 2 * T0>(gs);
        else zpass_launch1<N, 0>(gs);
    }
    // z FFT, Green multiply and inverse z FFT of the plane spectra (FP32)
    int green_z(double gs) {
        if constexpr (sizeof(T) == 4) {
            switch (mf.n) {
                case 64: CONAN_TIMED(prof, "green", st, zpass_launch<64>((float)gs)); break;
                case 128: CONAN_TIMED(prof, "green", st, zpass_launch<128>((float)gs)); break;
                case 256: CONAN_TIMED(prof, "green", st, zpass_launch<256>((float)gs)); break;
                case 512: CONAN_TIMED(prof, "green", st, zpass_launch<512>((float)gs)); break;
                default: CONAN_TIMED(prof, "green", st, zpass_launch<1024>((float)gs)); break;
            }
            return CONAN_OK;
        } else {
            return set_error(CONAN_ERR_UNSUPPORTED, "the z pass is FP32 only");
        }
    }

    // Plane transforms by thread-block clusters (fft_plane.cuh; FP32 3D,
    // n = 256 or 512, Lagrangian deposit): the forward pass reads the
    // accumulator mesh directly, so the step's density is never written.
    // plane_use: the autotuner's choice between them and cuFFT's planes.
    bool plane = false, plane_use = false;
    bool plane_inv = true;  // the inverse too (else cuFFT's 2D C2R after the z pass)
    bool plane_clear = PLANE_CLEAR;  // the forward pass clears the accumulator (else a memset)
    bool plane_on() const { return plane && plane_use && zpass && lag_on(); }
    int plane_kc = 16;       // kx columns per CTA of the plane pass
    unsigned plane_kcs = 0;  // the column counts that launch here (bit 0: 16, bit 1: 32)
    int plane_setup() {
        if constexpr (sizeof(T) == 4 && R == 3) {
            // CONAN_PLANE_PASS: 0 never, 1 both passes from the start, 2 the
            // forward pass from the start (else the default below, until the
            // autotuner decides)
            const char *pp = getenv("CONAN_PLANE_PASS");
            if (pp && *pp == '0') return CONAN_OK;
            // both column counts (clusters of 8 and of 16 CTAs at n = 512)
            // where they launch; the autotuner times both
            if (mf.n == 512) {
                CONAN_TRY((plane_setup_n<512, 32>()));
                CONAN_TRY((plane_setup_n<512, 16>()));
            }
            if (mf.n == 256) {
                CONAN_TRY((plane_setup_n<256, 32>()));
                CONAN_TRY((plane_setup_n<256, 16>()));
            }
            if (!plane) return CONAN_OK;
            // 32 columns per CTA: at 512^3 0.67 ms per forward pass against 0.69
            // with 16 (and 0.70 against 0.81 per inverse pass)
            if (plane_kcs & 2u) plane_kc = 32;
            const char *kc = getenv("CONAN_PLANE_COLUMNS");
            if (kc && atoi(kc) == 16 && (plane_kcs & 1u)) plane_kc = 16;
            if (kc && atoi(kc) == 32 && (plane_kcs & 2u)) plane_kc = 32;
            if (pp && (*pp == '1' || *pp == '2')) {
                plane_use = true;
                plane_inv = *pp == '1';  // 2: the forward pass only
            } else {
                // measured at 512^3: the forward pass here, cuFFT's inverse
                // (5.82 against 5.99 ms per step); elsewhere the autotuner decides
                plane_use = mf.n == 512;
                plane_inv = false;
            }
        }
        return CONAN_OK;
    }
    // On when both kernels launch in clusters of PlaneT::C CTAs on this GPU.
    template <int N, int KC> int plane_setup_n() {
        typedef PlaneT<N, KC> PT;
        if constexpr (PT::OK) {
            auto fk = k_plane_fwd<N, KC>;
            auto ik = k_plane_inv<N, KC>;
            if (!raise_dyn_smem(fk, PT::SMEM) || !raise_dyn_smem(ik, PT::SMEM)) return CONAN_OK;
            if (PT::C > 8 && (cudaFuncSetAttribute(fk, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
                              cudaFuncSetAttribute(ik, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
                cudaGetLastError();
                return CONAN_OK;
            }
            cudaLaunchConfig_t cfg = plane_cfg<N, KC>();
            cudaLaunchAttribute at;
            plane_cluster(cfg, at);
            int nc = 0;
            if (cudaOccupancyMaxActiveClusters(&nc, fk, &cfg) != cudaSuccess || nc < 1 ||
                cudaOccupancyMaxActiveClusters(&nc, ik, &cfg) != cudaSuccess || nc < 1) {
                cudaGetLastError();
                return CONAN_OK;
            }
            plane = true;
            plane_kc = KC;
            plane_kcs |= KC == 16 ? 1u : 2u;
        }
        return CONAN_OK;
    }
    template <int N, int KC> cudaLaunchConfig_t plane_cfg() const {
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)PlaneT<N, KC>::C, (unsigned)mf.n, (unsigned)mf.batch);
        cfg.blockDim = dim3((unsigned)PlaneT<N, KC>::THREADS);
        cfg.dynamicSmemBytes = PlaneT<N, KC>::SMEM;
        cfg.stream = st;
        return cfg;
    }
    static void plane_cluster(cudaLaunchConfig_t &cfg, cudaLaunchAttribute &at) {
        at.id = cudaLaunchAttributeClusterDimension;
        at.val.clusterDim.x = cfg.gridDim.x;
        at.val.clusterDim.y = 1;
        at.val.clusterDim.z = 1;
        cfg.attrs = &at;
        cfg.numAttrs = 1;
    }
    // 23 - log2(mass) when the particle mass is a power of two 2^e with
    // 0 <= e <= 23 (the mesh factor f is a power of two), else -1
    int plane_unit() const {
        int e = 0;
        const double fm = std::frexp(mass, &e);  // mass = fm 2^e, fm in [0.5, 1)
        if (fm != 0.5 || e - 1 < 0 || e - 1 > 23) return -1;
        return 23 - (e - 1);
    }
    template <int N, int KC> int plane_run(double gs) {
        if constexpr (sizeof(T) == 4 && PlaneT<N, KC>::OK) {
            cudaLaunchConfig_t cfg = plane_cfg<N, KC>();
            cudaLaunchAttribute at;
            plane_cluster(cfg, at);
            float2 *sp = reinterpret_cast<float2 *>(spec);
            CONAN_TIMED(prof, "plane_r2c", st,
                        CONAN_CUDA(cudaLaunchKernelEx(&cfg, k_plane_fwd<N, KC>, lacc, sp, mf, 0x1p-23 * mass,
                                                      (const float2 *)ztw, plane_clear ? 1 : 0, plane_unit())));
            if (!plane_clear)
                CONAN_TIMED(prof, "deposit_clear", st,
                            CONAN_CUDA(cudaMemsetAsync(lacc, 0, mf.cells * sizeof(unsigned long long), st)));
            CONAN_TRY(green_z(gs));
            if (plane_inv)
                CONAN_TIMED(prof, "plane_c2r", st,
                            CONAN_CUDA(cudaLaunchKernelEx(&cfg, k_plane_inv<N, KC>, (const float2 *)sp, (float *)mesh,
                                                          mf, (const float2 *)ztw)));
            else
                CONAN_TIMED(prof, "fft_c2r", st, CONAN_TRY(fft2.inverse(spec, mesh)));
            return CONAN_OK;
        } else {
            return set_error(CONAN_ERR_UNSUPPORTED, "no plane pass for this mesh");
        }
    }

    // The deposit of the current positions and the Poisson solve of the
    // kick that follows it: through the cluster plane pass when it is on,
    // else deposit() (density mesh) and poisson().
    int deposit_poisson(double a) {
        if (plane_on()) {
            CONAN_TRY(lag_accumulate());
            const double gs = poisson_scale(a);
            if (mf.n == 512) CONAN_TRY((plane_kc == 16 ? plane_run<512, 16>(gs) : plane_run<512, 32>(gs)));
            else CONAN_TRY((plane_kc == 16 ? plane_run<256, 16>(gs) : plane_run<256, 32>(gs)));
            CONAN_TRY(fd_gradient(mesh, grad));
            mesh_holds = 2;
            return CONAN_OK;
        }
        CONAN_TRY(deposit());
        return poisson(a);
    }

    // Green's function factor of a kick at a, with the per-member
    // normalisation 1 / (cells of one box).
    double poisson_scale(double a) const {
        return -G / (a * (double)((size_t)1 << mf.cshift)) * std::pow(prm.size / (2 * M_PI), 2);
    }

    int poisson(double a) {
        const double gs = poisson_scale(a);
        if (zpass) {
            // 2D R2C of every z plane, z pass with the Green multiply, 2D C2R
            if constexpr (sizeof(T) == 4) {
                CONAN_TIMED(prof, "fft_r2c", st, CONAN_TRY(fft2.forward(mesh, spec)));
                CONAN_TRY(green_z(gs));
                CONAN_TIMED(prof, "fft_c2r", st, CONAN_TRY(fft2.inverse(spec, mesh)));
                CONAN_TRY(fd_gradient(mesh, grad));
                mesh_holds = 2;
                return CONAN_OK;
            }
        }
        unsigned gb = (unsigned)((mf.spec + 255) / 256);
        CONAN_TIMED(prof, "fft_r2c", st, CONAN_TRY(fft.forward(mesh, spec)));
        CONAN_TRY(green(spec, gs));
        if (prm.gradient == CONAN_GRAD_SPECTRAL) {
            for (int k = 0; k < R; ++k) {
                CONAN_TIMED(prof, "spec_deriv", st, (k_spec_deriv<T><<<gb, 256, 0, st>>>(spec, spec2, mf, k)));
                CONAN_TIMED(prof, "fft_c2r", st, CONAN_TRY(fft.inverse(spec2, gm[k])));
            }
        }
        CONAN_TIMED(prof, "fft_c2r", st, CONAN_TRY(fft.inverse(spec, mesh)));
        if (prm.gradient == CONAN_GRAD_FD4) CONAN_TRY(fd_gradient(mesh, grad));
        mesh_holds = 2;
        return CONAN_OK;
    }

    // Packed FD4 gradient mesh of phi. (Measured at 512^3: the plain
    // thread-per-cell kernel beats four-cells-per-thread and warp-shuffle
    // variants, 0.64 against 0.68 and 0.83 ms.)
    // Gradient-mesh kernel: z-marching tiles (3D, 32 cells per side and
    // more) or one thread per cell in blocks of grad_block threads; the
    // autotuner picks one.
    bool grad_zm = FD_GRAD_ZM != 0;
    int grad_block = 256;
    bool grad_zm_fits() const { return R == 3 && mf.n >= 32; }

    int fd_gradient(const T *phi, G4<T> *g) {
        if constexpr (R == 3) {
            if (grad_zm && grad_zm_fits()) {
                const unsigned blocks = (unsigned)((size_t)(mf.n / 32) * (mf.n / 8) * (mf.n / FDZ_PLANES) * mf.batch);
                CONAN_TIMED(prof, "fd_grad", st, (k_fd_grad_zm<T><<<blocks, 256, 0, st>>>(phi, g, mf)));
                return CONAN_OK;
            }
        }
        const unsigned bs = (unsigned)grad_block;
        CONAN_TIMED(prof, "fd_grad", st,
                    (k_fd_grad<T, R><<<(unsigned)((mf.cells + bs - 1) / bs), bs, 0, st>>>(phi, g, mf)));
        return CONAN_OK;
    }

    // --- autotuner -----------------------------------------------------------
    // On the current particle state (a clustered one: tile costs grow as the
    // particles cluster) it chooses (1) the deposit: the sorted tile variants,
    // the Lagrangian window tiles V0..V2 and the direct two-cell window
    // (FP32); (2) the gradient-mesh kernel: one thread per cell in blocks of
    // 128, 256 or 512, or z-marching tiles. Knobs are tuned one after the
    // other; each candidate runs one untimed and TUNE_STEPS timed leapfrog
    // steps (CUDA events) from a copy of the state, which is restored at the
    // end.
    struct TuneRec {
        std::string knob, value;
        double ms;  // per timed step
        bool chosen;
    };
    std::vector<TuneRec> tuned;
    static constexpr int TUNE_STEPS = 2;
    struct DepCand {
        int mode;  // 0 sorted, 1 Lagrangian window, 2 Lagrangian direct, 3 Lagrangian window, persistent
        int v;
        std::string name;
    };

    template <int V> bool dep_fits() const {
        typedef DepTile<R, V> D;
        return mf.n >= D::TX && mf.n >= D::TY && mf.n >= D::TZ;
    }
    bool lag_set(int v, bool direct) {
        return v == 0 ? lag_try<0>(direct) : v == 1 ? lag_try<1>(direct) : lag_try<2>(direct);
    }
    int dep_apply(const DepCand &c) {
        CONAN_TRY(drop_lag_deposit());
        pers = c.mode == 3;
        if (c.mode == 0) {
            dep_variant = c.v;
            return CONAN_OK;
        }
        if (!lag_set(c.v, c.mode == 2)) return set_error(CONAN_ERR_STATE, "deposit candidate %s no longer fits", c.name.c_str());
        dep_variant = DEP_LAG;
        CONAN_TRY(tma_setup());
        return pers_setup();
    }

    // Time of one timed leapfrog step from the saved state.
    int tune_time(T *const *save, double a, double da, double *ms) {
        for (int k = 0; k < R; ++k) {
            CONAN_CUDA(cudaMemcpyAsync(P.d[k], save[k], np * sizeof(T), cudaMemcpyDeviceToDevice, st));
            CONAN_CUDA(cudaMemcpyAsync(P.p[k], save[R + k], np * sizeof(T), cudaMemcpyDeviceToDevice, st));
        }
        CONAN_TRY(positions_reset());
        double aa = a;
        CONAN_TRY(steps(aa, da, 0, 1));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        CONAN_CUDA(cudaEventCreate(&e0));
        CONAN_CUDA(cudaEventCreate(&e1));
        cudaEventRecord(e0, st);
        int rc = steps(aa, da, 1, 1 + TUNE_STEPS);
        cudaEventRecord(e1, st);
        cudaError_t se = cudaEventSynchronize(e1);
        float t = 0;
        if (se == cudaSuccess) se = cudaEventElapsedTime(&t, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc != CONAN_OK) return rc;
        if (se != cudaSuccess) return set_error(CONAN_ERR_CUDA, "autotuner timing: %s", cudaGetErrorString(se));
        *ms = t / TUNE_STEPS;
        return check_err();
    }

    int tune(double a, double da) {
        tuned.clear();
        const double apos = a_pos, amom = a_mom;
        std::vector<T *> save(2 * R, nullptr);
        for (auto &b : save) CONAN_CUDA(cudaMalloc(&b, np * sizeof(T)));
        for (int k = 0; k < R; ++k) {
            CONAN_CUDA(cudaMemcpyAsync(save[k], P.d[k], np * sizeof(T), cudaMemcpyDeviceToDevice, st));
            CONAN_CUDA(cudaMemcpyAsync(save[R + k], P.p[k], np * sizeof(T), cudaMemcpyDeviceToDevice, st));
        }
        const bool prof_was = prof.on;
        prof.on = false;
        int rc = tune_knobs(save.data(), a, da);
        prof.on = prof_was;
        for (int k = 0; k < R && rc == CONAN_OK; ++k) {
            cudaMemcpyAsync(P.d[k], save[k], np * sizeof(T), cudaMemcpyDeviceToDevice, st);
            cudaMemcpyAsync(P.p[k], save[R + k], np * sizeof(T), cudaMemcpyDeviceToDevice, st);
        }
        cudaStreamSynchronize(st);
        for (auto b : save) cudaFree(b);
        if (rc != CONAN_OK) return rc;
        CONAN_TRY(positions_reset());
        mesh_holds = 0;
        a_pos = apos;
        a_mom = amom;
        return CONAN_OK;
    }

    int tune_knobs(T *const *save, double a, double da) {
        // (1) the deposit
        std::vector<DepCand> cands;
        if (dep_fits<0>()) cands.push_back({0, 0, "sorted 32x8x8 / 256 threads"});
        if (dep_fits<1>()) cands.push_back({0, 1, "sorted 32x4x8 / 128 threads"});
        if (dep_fits<2>()) cands.push_back({0, 2, "sorted 32x16x8 / 512 threads"});
        if (sizeof(T) == 4 && lacc) {
            const char *tile[3] = {"", "", ""};
            if (R == 3) tile[0] = "32x8x8", tile[1] = "16x8x8", tile[2] = "8x8x8";
            if (R == 2) tile[0] = "64x32", tile[1] = "32x16", tile[2] = "16x16";
            if (R == 1) tile[0] = "2048", tile[1] = "512", tile[2] = "128";
            for (int v = 0; v < 3; ++v)
                if (lag_set(v, false)) cands.push_back({1, v, std::string("lagrangian window, tile ") + tile[v]});
            if (R == 3)
                for (int v = 0; v < 2; ++v)
                    if (lag_set(v, false))
                        cands.push_back({3, v, std::string("lagrangian window, tile ") + tile[v] + ", persistent"});
            for (int v = 0; v < 3; ++v)
                if (lag_set(v, true)) {
                    cands.push_back({2, v, std::string("lagrangian direct, tile ") + tile[v]});
                    break;
                }
        }
        int best = -1;
        double bms = 1e30;
        for (size_t i = 0; i < cands.size(); ++i) {
            double ms = 0;
            CONAN_TRY(dep_apply(cands[i]));
            CONAN_TRY(tune_time(save, a, da, &ms));
            tuned.push_back({"deposit", cands[i].name, ms, false});
            if (ms < bms) bms = ms, best = (int)i;
        }
        if (best >= 0) {
            CONAN_TRY(dep_apply(cands[best]));
            tuned[tuned.size() - cands.size() + best].chosen = true;
        }
        // (2) the gradient mesh (FD4 only)
        if (prm.gradient == CONAN_GRAD_FD4) {
            struct GC { bool zm; int block; std::string name; };
            std::vector<GC> g = {{false, 128, "thread per cell, 128"}, {false, 256, "thread per cell, 256"},
                                 {false, 512, "thread per cell, 512"}};
            if (grad_zm_fits()) g.push_back({true, 256, "z-marching 32x8 tiles"});
            best = -1;
            bms = 1e30;
            for (size_t i = 0; i < g.size(); ++i) {
                grad_zm = g[i].zm;
                grad_block = g[i].block;
                double ms = 0;
                CONAN_TRY(tune_time(save, a, da, &ms));
                tuned.push_back({"gradient", g[i].name, ms, false});
                if (ms < bms) bms = ms, best = (int)i;
            }
            grad_zm = g[best].zm;
            grad_block = g[best].block;
            tuned[tuned.size() - g.size() + best].chosen = true;
        }
        // (3) the z pass's lines per CTA (FP32 3D plane-transform solve)
        if (zpass) {
            const std::vector<int> w = zpass_widths();
            best = -1;
            bms = 1e30;
            for (size_t i = 0; i < w.size(); ++i) {
                ztx = w[i];
                double ms = 0;
                CONAN_TRY(tune_time(save, a, da, &ms));
                char nm[64];
                if (w[i]) snprintf(nm, sizeof nm, "%d lines per CTA", w[i]);
                else snprintf(nm, sizeof nm, "default lines per CTA");
                tuned.push_back({"z pass", nm, ms, false});
                if (ms < bms) bms = ms, best = (int)i;
            }
            ztx = w[best];
            tuned[tuned.size() - w.size() + best].chosen = true;
        }
        // (4) the x and y transforms of the planes: thread-block clusters or
        // cuFFT's 2D plans
        if (plane && lag_on()) {
            struct PC { bool use, inv; int kc; std::string name; };
            std::vector<PC> pc = {{false, true, plane_kc, "cuFFT 2D plans"}};
            for (int kc : {16, 32})
                if (plane_kcs & (kc == 16 ? 1u : 2u)) {
                    const std::string cl = "thread-block clusters of " + std::to_string(mf.n / (2 * kc)) + " CTAs, " +
                                           std::to_string(kc) + " columns each";
                    pc.push_back({true, true, kc, cl});
                    pc.push_back({true, false, kc, cl + " (forward; cuFFT inverse)"});
                }
            best = -1;
            bms = 1e30;
            for (size_t i = 0; i < pc.size(); ++i) {
                plane_use = pc[i].use;
                plane_inv = pc[i].inv;
                plane_kc = pc[i].kc;
                double ms = 0;
                CONAN_TRY(tune_time(save, a, da, &ms));
                tuned.push_back({"plane transforms", pc[i].name, ms, false});
                if (ms < bms) bms = ms, best = (int)i;
            }
            plane_use = pc[best].use;
            plane_inv = pc[best].inv;
            plane_kc = pc[best].kc;
            tuned[tuned.size() - pc.size() + best].chosen = true;
        }
        return CONAN_OK;
    }

    std::string tune_report() const {
        std::string s = "[";
        for (size_t i = 0; i < tuned.size(); ++i) {
            char buf[256];
            snprintf(buf, sizeof buf, "%s{\"knob\": \"%s\", \"value\": \"%s\", \"ms_per_step\": %.4f, \"chosen\": %s}",
                     i ? ", " : "", tuned[i].knob.c_str(), tuned[i].value.c_str(), tuned[i].ms,
                     tuned[i].chosen ? "true" : "false");
            s += buf;
        }
        return s + "]";
    }

    int autotune(double a, double da, char *report, size_t len) override {
        CONAN_TRY(tune(a, da));
        if (report && len) {
            std::string r = tune_report();
            std::strncpy(report, r.c_str(), len - 1);
            report[len - 1] = 0;
            if (r.size() >= len) return set_error(CONAN_ERR_ARG, "report buffer too small (%zu bytes needed)", r.size() + 1);
        }
        return CONAN_OK;
    }

    // Kick and/or drift of every particle. rank_after: prepare the next
    // deposit (counting-sort ranks, or with the Lagrangian deposit and a
    // drift, the deposit itself in the same kernel).
    int gkd(bool kick, double ck, bool drift, double cd, bool rank_after) {
        const bool fuse = rank_after && drift && lag_on() && prm.gradient == CONAN_GRAD_FD4;
        rank_after = rank_after && !lag_on();  // the Lagrangian deposit needs no ranks
        // ranks of positions about to move are stale either way
        if ((rank_after || drift) && ranks_pending) {
            CONAN_CUDA(cudaMemsetAsync(count, 0, mf.cells * sizeof(uint32_t), st));
            ranks_pending = false;
        }
        if (drift) CONAN_TRY(drop_lag_deposit());
        GKD c{ck, cd, kick ? 1 : 0, drift ? 1 : 0, rank_after ? 1 : 0, prm.periodic_gather ? 1 : 0};
        const char *name = kick ? (drift ? "gather_kick_drift" : "gather_kick") : "drift";
        if (fuse) {
            const char *fname = kick ? "gather_kick_drift_deposit" : "drift_deposit";
            if (lag_v == 0) CONAN_TRY(launch_gkd_lag<0>(c, fname));
            else if (lag_v == 1) CONAN_TRY(launch_gkd_lag<1>(c, fname));
            else CONAN_TRY(launch_gkd_lag<2>(c, fname));
            lag_ready = true;
            return CONAN_OK;
        }
        // the last kick of a run (no drift, no deposit) on the same staged
        // tiles instead of the thread-per-particle kernel
        if (kick && !drift && !rank_after && lag_on() && prm.gradient == CONAN_GRAD_FD4) {
            c.deposit = 0;
            if (lag_v == 0) CONAN_TRY(launch_gkd_lag<0>(c, name));
            else if (lag_v == 1) CONAN_TRY(launch_gkd_lag<1>(c, name));
            else CONAN_TRY(launch_gkd_lag<2>(c, name));
            return CONAN_OK;
        }
        if (prm.gradient == CONAN_GRAD_SPECTRAL)
            CONAN_TIMED(prof, name, st,
                        (k_gkd<T, R, true><<<grid_p(), 256, 0, st>>>(P, mf, mesh, gm[0], gm[1], gm[2], grad, c,
                                                                     count, rank)));
        else
            CONAN_TIMED(prof, name, st,
                        (k_gkd<T, R, false><<<grid_p(), 256, 0, st>>>(P, mf, mesh, gm[0], gm[1], gm[2], grad, c,
                                                                      count, rank)));
        if (rank_after) ranks_pending = true;
        return CONAN_OK;
    }

    double coef_drift(double a, double da) const {
        return da / (a * a * adot(prm.H0, prm.Omega_m, prm.Omega_L, a));
    }
    double coef_kick(double a, double da) const {
        return (da / adot(prm.H0, prm.Omega_m, prm.Omega_L, a)) / (res_f * res_f);
    }

    // --- API ---------------------------------------------------------------
    int init(const double *phi, double apos, double amom) override {
        if (!phi) return set_error(CONAN_ERR_ARG, "null potential");
        CONAN_TRY(upload_mesh(phi, mesh, mm.cells));
        double cdz = -apos / (res_m * res_f), cpz = -amom / (res_m * res_f);
        CONAN_TIMED(prof, "zeldovich", st, (k_zeldovich<T, R><<<grid_p(), 256, 0, st>>>(P, mesh, mm, cdz, cpz)));
        CONAN_TRY(positions_reset());
        mesh_holds = 0;
        a_pos = apos;
        a_mom = amom;
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }

    int drift(double a, double da) override {
        CONAN_TRY(gkd(false, 0, true, coef_drift(a, da), true));
        a_pos = a;
        return CONAN_OK;
    }

    int kick(double a, double da) override {
        CONAN_TRY(deposit_poisson(a));
        CONAN_TRY(gkd(true, coef_kick(a, da), false, 0, false));
        a_mom = a;
        return CONAN_OK;
    }

    // Steps [i0, i1) of a leapfrog run starting at a(i0) = a; the first
    // drift is separate, every later drift is fused into the previous kick.
    int steps(double &a, double da, unsigned i0, unsigned i1) {
        CONAN_TRY(gkd(false, 0, true, coef_drift(a, da), true));
        a_pos = a;
        for (unsigned i = i0; i < i1; ++i) {
            double am = a + da / 2;
            CONAN_TRY(deposit_poisson(am));
            bool last = i + 1 == i1;
            double an = a + da;
            CONAN_TRY(gkd(true, coef_kick(am, da), !last, last ? 0 : coef_drift(an, da), !last));
            a_mom = am;
            a = an;
            if (!last) a_pos = a;
        }
        return CONAN_OK;
    }

    // The instantiated graph of the last run segment. A later segment of the
    // same shape (the same launches with other scale-factor coefficients)
    // updates it in place instead of instantiating a new one.
    cudaGraphExec_t gexec = nullptr;

    // Steps [i0, i1) captured into a CUDA graph and launched; returns after
    // the graph has run.
    int graph_segment(double &a, double da, unsigned i0, unsigned i1) {
        cudaGraph_t g = nullptr;
        CONAN_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int rc = steps(a, da, i0, i1);
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        if (rc != CONAN_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (ce != cudaSuccess) return set_error(CONAN_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        bool updated = false;
        if (gexec) {
            cudaGraphExecUpdateResultInfo info{};
            if (cudaGraphExecUpdate(gexec, g, &info) == cudaSuccess) {
                updated = true;
            } else {  // another shape: instantiate anew
                cudaGetLastError();
                cudaGraphExecDestroy(gexec);
                gexec = nullptr;
            }
        }
        cudaError_t ie = updated ? cudaSuccess : cudaGraphInstantiate(&gexec, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            gexec = nullptr;
            return set_error(CONAN_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(ie));
        }
        cudaError_t le = cudaGraphLaunch(gexec, st);
        cudaError_t se = cudaStreamSynchronize(st);
        if (le != cudaSuccess) return set_error(CONAN_ERR_CUDA, "graph launch failed: %s", cudaGetErrorString(le));
        if (se != cudaSuccess) return set_error(CONAN_ERR_CUDA, "graph execution failed: %s", cudaGetErrorString(se));
        return CONAN_OK;
    }

    int run(conan_pm *h, const double *phi, double a0, double da, unsigned n, conan_step_cb cb,
            void *user) override {
        if (phi) CONAN_TRY(init(phi, a0, a0 + da / 2));
        double a = a0;
        unsigned i = 0;
        while (i < n) {
            unsigned seg_end = n;
            if (cb) {
                unsigned k = cb_every ? cb_every : 1;
                seg_end = ((i / k) + 1) * k;
                if (seg_end > n) seg_end = n;
            }
            if (!prof.on && !debug_sync()) {
                CONAN_TRY(graph_segment(a, da, i, seg_end));
            } else {
                CONAN_TRY(steps(a, da, i, seg_end));
            }
            i = seg_end;
            if (cb) {
                CONAN_CUDA(cudaStreamSynchronize(st));
                if (cb(h, i - 1, a, user) != 0)
                    return set_error(CONAN_ERR_STATE, "step callback stopped the run after step %u", i - 1);
            }
        }
        CONAN_CUDA(cudaStreamSynchronize(st));
        return check_err();
    }

    // Reads and clears the kernels' self-check word.
    int check_err() {
        int h = 0;
        CONAN_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        CONAN_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        CONAN_CUDA(cudaStreamSynchronize(st));
        return err_word_status(h);
    }

    int get_state(double *X, double *Pm) override {
        CONAN_TRY(export_state(P, np, X, Pm));
        return check_err();
    }

    int set_state(const double *X, const double *Pm, double apos, double amom) override {
        if (!X || !Pm) return set_error(CONAN_ERR_ARG, "null state");
        const size_t cp = stage_particles();
        for (size_t i0 = 0; i0 < np; i0 += cp) {
            const size_t cnt = std::min(cp, np - i0);
            CONAN_CUDA(cudaMemcpyAsync(stage[0], X + i0 * R, cnt * R * sizeof(double), cudaMemcpyHostToDevice, st));
            CONAN_CUDA(cudaMemcpyAsync(stage[1], Pm + i0 * R, cnt * R * sizeof(double), cudaMemcpyHostToDevice, st));
            CONAN_TIMED(prof, "import", st,
                        (k_import<T, R><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(P, res_f, i0, cnt, stage[0],
                                                                                       stage[1])));
        }
        CONAN_TRY(positions_reset());
        a_pos = apos;
        a_mom = amom;
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }

    int mesh_out(double *out) {
        for (size_t c0 = 0, b = 0; c0 < mf.cells; c0 += stage_n, b ^= 1) {
            const size_t cnt = std::min(stage_n, mf.cells - c0);
            CONAN_TIMED(prof, "convert", st,
                        (k_convert<T, double><<<(unsigned)((cnt + 255) / 256), 256, 0, st>>>(mesh + c0, stage[b], cnt,
                                                                                          1.0, 0.0)));
            CONAN_CUDA(cudaMemcpyAsync(out + c0, stage[b], cnt * sizeof(double), cudaMemcpyDeviceToHost, st));
        }
        CONAN_CUDA(cudaStreamSynchronize(st));
        return check_err();
    }

    int density(double *out) override {
        CONAN_TRY(deposit());
        return mesh_out(out);
    }

    int potential(double *out) override {
        if (mesh_holds != 2) return set_error(CONAN_ERR_STATE, "no potential: call kick first");
        return mesh_out(out);
    }

    int power_spectrum(int nbins, double *k, double *Pk, double *cnt) override {
        if (nbins < 1) return set_error(CONAN_ERR_ARG, "nbins must be positive");
        CONAN_TRY(deposit());
        CONAN_TIMED(prof, "fft_r2c", st, CONAN_TRY(fft.forward(mesh, spec)));
        mesh_holds = 1;
        CONAN_TRY(spectrum_bins<T>(spec, mf, prm.size, nbins, k, Pk, cnt, st, this));
        return check_err();
    }

    int scale_factors(double *ap, double *am) override {
        if (ap) *ap = a_pos;
        if (am) *am = a_mom;
        return CONAN_OK;
    }
    int set_profiling(int on) override {
        prof.on = on != 0;
        return CONAN_OK;
    }
    int profile_entry(int i, char *name, int *launches, double *ms) override {
        CONAN_CUDA(cudaStreamSynchronize(st));
        CONAN_TRY(prof.collect());
        if (i < 0 || i >= (int)prof.names.size()) return set_error(CONAN_ERR_ARG, "no profile entry %d", i);
        if (name) {
            std::strncpy(name, prof.names[i].c_str(), 63);
            name[63] = 0;
        }
        if (launches) *launches = prof.launches[i];
        if (ms) *ms = prof.total_ms[i];
        return CONAN_OK;
    }
    int profile_reset() override {
        CONAN_CUDA(cudaStreamSynchronize(st));
        CONAN_TRY(prof.collect());
        prof.reset();
        return CONAN_OK;
    }
    int device_bytes(size_t *b) override {
        *b = bytes + fft.work_bytes * 0;
        return CONAN_OK;
    }
    int sync() override {
        CONAN_CUDA(cudaStreamSynchronize(st));
        return check_err();
    }
    int set_cb_every(unsigned k) override {
        cb_every = k ? k : 1;
        return CONAN_OK;
    }
    int device() const override { return prm.device; }
    void *stream() const override { return (void *)st; }
};

// Power-spectrum bins from a half spectrum (deterministic two-level sum).
__global__ void k_pk_final(const double *__restrict__ part, int nblocks, int nbins, double L, int R,
                           double ncells, double *__restrict__ out) {
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 3 * nbins) return;
    double s = 0;
    for (int b = 0; b < nblocks; ++b) s += part[(size_t)b * 3 * nbins + j];
    out[j] = s;
}

template <typename T>
int spectrum_bins(const typename Cplx<T>::type *spec, const Mesh &m, double L, int nbins, double *k,
                  double *Pk, double *cnt, cudaStream_t st, PMBase *) {
    const int threads = 256, nblocks = 148 * 2;
    size_t sh = (size_t)(threads / 32) * 3 * nbins * sizeof(double);
    if (sh > 200 * 1024) return set_error(CONAN_ERR_ARG, "too many bins (%d)", nbins);
    double *part = nullptr, *out = nullptr;
    CONAN_CUDA(cudaMallocAsync((void **)&part, (size_t)nblocks * 3 * nbins * sizeof(double), st));
    CONAN_CUDA(cudaMallocAsync((void **)&out, 3 * (size_t)nbins * sizeof(double), st));
    if (sh > 48 * 1024)
        CONAN_CUDA(cudaFuncSetAttribute(k_pk_partial<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh));
    k_pk_partial<T><<<nblocks, threads, sh, st>>>(spec, m, nbins, part);
    CONAN_LAUNCHED();
    k_pk_final<<<(3 * nbins + 255) / 256, 256, 0, st>>>(part, nblocks, nbins, L, m.R, (double)m.cells, out);
    CONAN_LAUNCHED();
    std::vector<double> h(3 * (size_t)nbins);
    CONAN_CUDA(cudaMemcpyAsync(h.data(), out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    CONAN_CUDA(cudaFreeAsync(part, st));
    CONAN_CUDA(cudaFreeAsync(out, st));
    CONAN_CUDA(cudaStreamSynchronize(st));
    double norm = std::pow(L, m.R) / ((double)m.cells * (double)m.cells);
    for (int b = 0; b < nbins; ++b) {
        double c = h[2 * nbins + b];
        if (cnt) cnt[b] = c;
        if (k) k[b] = c > 0 ? h[nbins + b] / c * 2 * M_PI / L : 0;
        if (Pk) Pk[b] = c > 0 ? h[b] / c * norm : 0;
    }
    return CONAN_OK;
}

template int spectrum_bins<float>(const cufftComplex *, const Mesh &, double, int, double *, double *,
                                  double *, cudaStream_t, PMBase *);
template int spectrum_bins<double>(const cufftDoubleComplex *, const Mesh &, double, int, double *,
                                   double *, double *, cudaStream_t, PMBase *);

}  // namespace conan

#include "adjoint_impl.cuh"
#include "ensemble_impl.cuh"

namespace conan {

PMBase *make_pm(const conan_pm_params &p) {
    PMBase *b = nullptr;
    int rc = CONAN_OK;
#define MAKE(T, R)                     \
    {                                  \
        auto *x = new PM<T, R>();      \
        rc = x->create(p);             \
        b = x;                         \
    }
    if (p.precision == CONAN_FP32) {
        if (p.dim == 1) MAKE(float, 1) else if (p.dim == 2) MAKE(float, 2) else MAKE(float, 3)
    } else {
        if (p.dim == 1) MAKE(double, 1) else if (p.dim == 2) MAKE(double, 2) else MAKE(double, 3)
    }
#undef MAKE
    if (rc != CONAN_OK) {
        std::string msg = last_error();
        delete b;
        last_error() = msg;
        return nullptr;
    }
    return b;
}

}  // namespace conan

using namespace conan;

namespace conan {

// One CTA waits on a shared-memory barrier that nothing completes, with the
// bounded wait of the staged kernels; the wait must run out (bit 3).
__global__ void k_wait_selftest(int *err, unsigned polls) {
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0 && !tma_wait(&bar, polls)) atomicOr(err, 8);
}

}  // namespace conan

struct conan_pm {
    PMBase *impl;
};

#define H_GUARD(h)                                                       \
    do {                                                                 \
        if (!(h) || !(h)->impl) return set_error(CONAN_ERR_ARG, "null handle"); \
        CONAN_TRY(device_guard((h)->impl->device()));                    \
    } while (0)

extern "C" {

const char *conan_last_error(void) { return last_error().c_str(); }
const char *conan_version(void) { return "conan_b200 1.0 (sm_100a)"; }

int conan_device_count(int *n) {
    if (!n) return set_error(CONAN_ERR_ARG, "null pointer");
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        c = 0;
    }
    *n = c;
    return CONAN_OK;
}

int conan_selftest_bounded_wait(unsigned polls, void *stream) {
    int dev = 0;
    CONAN_CUDA(cudaGetDevice(&dev));
    CONAN_TRY(device_guard(dev));
    cudaStream_t st = (cudaStream_t)stream;
    int *err = nullptr, h = 0;
    CONAN_CUDA(cudaMalloc(&err, sizeof(int)));
    cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e == cudaSuccess) {
        k_wait_selftest<<<1, 32, 0, st>>>(err, polls);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(err);
    if (e != cudaSuccess) return set_error(CONAN_ERR_CUDA, "bounded-wait self-test: %s", cudaGetErrorString(e));
    return err_word_status(h);
}

conan_pm *conan_pm_create(const conan_pm_params *p) {
    last_error().clear();
    if (check_pm_params(p) != CONAN_OK) return nullptr;
    if (device_guard(p->device) != CONAN_OK) return nullptr;
    PMBase *b = make_pm(*p);
    if (!b) return nullptr;
    return new conan_pm{b};
}

void conan_pm_destroy(conan_pm *h) {
    if (!h) return;
    if (h->impl) {
        cudaSetDevice(h->impl->device());
        delete h->impl;
    }
    delete h;
}

int conan_pm_init(conan_pm *h, const double *phi, double a_pos, double a_mom) {
    H_GUARD(h);
    return h->impl->init(phi, a_pos, a_mom);
}
int conan_pm_drift(conan_pm *h, double a, double da) {
    H_GUARD(h);
    return h->impl->drift(a, da);
}
int conan_pm_kick(conan_pm *h, double a, double da) {
    H_GUARD(h);
    return h->impl->kick(a, da);
}
int conan_pm_set_callback_interval(conan_pm *h, unsigned k) {
    H_GUARD(h);
    return h->impl->set_cb_every(k);
}
int conan_pm_set_deposit(conan_pm *h, int mode) {
    H_GUARD(h);
    return h->impl->set_deposit(mode);
}
int conan_pm_get_deposit(conan_pm *h, int *mode) {
    H_GUARD(h);
    return h->impl->get_deposit(mode);
}
int conan_pm_run(conan_pm *h, const double *phi, double a0, double da, unsigned n, conan_step_cb cb,
                 void *user) {
    H_GUARD(h);
    return h->impl->run(h, phi, a0, da, n, cb, user);
}
int conan_pm_get_state(conan_pm *h, double *X, double *P) {
    H_GUARD(h);
    return h->impl->get_state(X, P);
}
int conan_pm_set_state(conan_pm *h, const double *X, const double *P, double a_pos, double a_mom) {
    H_GUARD(h);
    return h->impl->set_state(X, P, a_pos, a_mom);
}
int conan_pm_scale_factors(conan_pm *h, double *a_pos, double *a_mom) {
    H_GUARD(h);
    return h->impl->scale_factors(a_pos, a_mom);
}
int conan_pm_density(conan_pm *h, double *delta_out) {
    H_GUARD(h);
    if (!delta_out) return set_error(CONAN_ERR_ARG, "null output");
    return h->impl->density(delta_out);
}
int conan_pm_potential(conan_pm *h, double *phi_out) {
    H_GUARD(h);
    if (!phi_out) return set_error(CONAN_ERR_ARG, "null output");
    return h->impl->potential(phi_out);
}
int conan_pm_power_spectrum(conan_pm *h, int nbins, double *k, double *P, double *count) {
    H_GUARD(h);
    return h->impl->power_spectrum(nbins, k, P, count);
}
int conan_pm_set_profiling(conan_pm *h, int enable) {
    H_GUARD(h);
    return h->impl->set_profiling(enable);
}
int conan_pm_profile_entry(conan_pm *h, int i, char *name, int *launches, double *total_ms) {
    H_GUARD(h);
    return h->impl->profile_entry(i, name, launches, total_ms);
}
int conan_pm_profile_reset(conan_pm *h) {
    H_GUARD(h);
    return h->impl->profile_reset();
}
int conan_pm_device_bytes(conan_pm *h, size_t *bytes) {
    H_GUARD(h);
    if (!bytes) return set_error(CONAN_ERR_ARG, "null pointer");
    return h->impl->device_bytes(bytes);
}
int conan_pm_sync(conan_pm *h) {
    H_GUARD(h);
    return h->impl->sync();
}
int conan_pm_autotune(conan_pm *h, double a, double da, char *report, size_t len) {
    H_GUARD(h);
    if (!(da > 0) || !(a > 0)) return set_error(CONAN_ERR_ARG, "need a > 0 and da > 0");
    return h->impl->autotune(a, da, report, len);
}
int conan_pm_get_stream(conan_pm *h, void **stream) {
    H_GUARD(h);
    if (!stream) return set_error(CONAN_ERR_ARG, "null pointer");
    *stream = h->impl->stream();
    return CONAN_OK;
}

}  // extern "C"

struct conan_diff {
    DiffBase *impl;
};

extern "C" {

conan_diff *conan_diff_create(const conan_diff_params *p) {
    last_error().clear();
    if (!p) {
        set_error(CONAN_ERR_ARG, "null parameters");
        return nullptr;
    }
    if (check_pm_params(&p->pm) != CONAN_OK || check_ic_params(&p->ic) != CONAN_OK) return nullptr;
    if (p->ic.dim != p->pm.dim || (1 << p->ic.mbits) != p->pm.n_mass) {
        set_error(CONAN_ERR_ARG, "ic and pm parameters disagree on dim / particles per side");
        return nullptr;
    }
    if (p->pm.gradient != CONAN_GRAD_FD4) {
        set_error(CONAN_ERR_UNSUPPORTED, "the adjoint supports the FD4 gradient only");
        return nullptr;
    }
    if (p->n < 1 || !(p->da > 0) || !(p->a0 > 0)) {
        set_error(CONAN_ERR_ARG, "need n >= 1, a0 > 0, da > 0");
        return nullptr;
    }
    if (device_guard(p->pm.device) != CONAN_OK) return nullptr;
    DiffBase *b = make_diff(*p);
    if (!b) return nullptr;
    return new conan_diff{b};
}

void conan_diff_destroy(conan_diff *h) {
    if (!h) return;
    if (h->impl) {
        cudaSetDevice(h->impl->device());
        delete h->impl;
    }
    delete h;
}

int conan_diff_forward(conan_diff *h, const void *noise_dev, void *density_out_dev, void *stream) {
    if (!h || !h->impl) return set_error(CONAN_ERR_ARG, "null handle");
    if (!noise_dev || !density_out_dev) return set_error(CONAN_ERR_ARG, "null buffer");
    CONAN_TRY(device_guard(h->impl->device()));
    return h->impl->forward(noise_dev, density_out_dev, stream);
}

int conan_diff_backward(conan_diff *h, const void *grad_density_dev, void *grad_noise_dev, void *stream) {
    if (!h || !h->impl) return set_error(CONAN_ERR_ARG, "null handle");
    if (!grad_density_dev || !grad_noise_dev) return set_error(CONAN_ERR_ARG, "null buffer");
    CONAN_TRY(device_guard(h->impl->device()));
    return h->impl->backward(grad_density_dev, grad_noise_dev, stream);
}

}  // extern "C"

struct conan_ens {
    EnsBase *impl;
};

#define ENS_GUARD(h)                                                              \
    do {                                                                          \
        if (!(h) || !(h)->impl) return set_error(CONAN_ERR_ARG, "null handle");   \
        CONAN_TRY(device_guard((h)->impl->device()));                             \
    } while (0)

extern "C" {

conan_ens *conan_ens_create(const conan_ens_params *p, int n_members, const conan_ens_member *m) {
    last_error().clear();
    if (!p || !m || n_members < 1) {
        set_error(CONAN_ERR_ARG, "need parameters and at least one member");
        return nullptr;
    }
    if (p->dim != 2 && p->dim != 3) {
        set_error(CONAN_ERR_UNSUPPORTED, "ensembles run in 2 or 3 dimensions");
        return nullptr;
    }
    if (p->n < 1 || !(p->a0 > 0) || !(p->da > 0) || !(p->H0 > 0) ||
        (p->precision != CONAN_FP32 && p->precision != CONAN_FP64)) {
        set_error(CONAN_ERR_ARG, "bad run parameters (n >= 1, a0, da, H0 > 0, precision)");
        return nullptr;
    }
    for (int i = 0; i < n_members; ++i)
        if (m[i].mbits < 3 || m[i].mbits > (p->dim == 3 ? 10 : 14) || !(m[i].size > 0)) {
            set_error(CONAN_ERR_ARG, "member %d: mbits %d / size %g out of range", i, m[i].mbits, m[i].size);
            return nullptr;
        }
    if (device_guard(p->device) != CONAN_OK) return nullptr;
    EnsBase *b = make_ens(*p, n_members, m);
    if (!b) return nullptr;
    return new conan_ens{b};
}

void conan_ens_destroy(conan_ens *h) {
    if (!h) return;
    if (h->impl) {
        cudaSetDevice(h->impl->device());
        delete h->impl;
    }
    delete h;
}

int conan_ens_init(conan_ens *h) {
    ENS_GUARD(h);
    return h->impl->init();
}
int conan_ens_run(conan_ens *h) {
    ENS_GUARD(h);
    return h->impl->run();
}
int conan_ens_forward_adjoint(conan_ens *h, double *loss_out) {
    ENS_GUARD(h);
    return h->impl->forward_adjoint(loss_out);
}
int conan_ens_power_spectrum(conan_ens *h, int member, int nbins, double *k, double *P, double *count) {
    ENS_GUARD(h);
    if (nbins < 1) return set_error(CONAN_ERR_ARG, "nbins must be positive");
    return h->impl->power_spectrum(member, nbins, k, P, count);
}
int conan_ens_state(conan_ens *h, int member, double *X, double *P) {
    ENS_GUARD(h);
    return h->impl->state(member, X, P);
}
int conan_ens_member_fields(conan_ens *h, int member, double *noise, double *target, double *gnoise) {
    ENS_GUARD(h);
    return h->impl->member_fields(member, noise, target, gnoise);
}
int conan_ens_last_ms(conan_ens *h, double *run_ms, double *adjoint_ms) {
    ENS_GUARD(h);
    return h->impl->last_ms(run_ms, adjoint_ms);
}
int conan_ens_total_particles(conan_ens *h, size_t *n) {
    ENS_GUARD(h);
    if (!n) return set_error(CONAN_ERR_ARG, "null pointer");
    *n = h->impl->total_particles();
    return CONAN_OK;
}
int conan_ens_describe(conan_ens *h, char *buf, size_t len) {
    ENS_GUARD(h);
    if (!buf || len == 0) return set_error(CONAN_ERR_ARG, "null buffer");
    std::string s = h->impl->describe();
    std::strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = 0;
    return s.size() < len ? CONAN_OK : set_error(CONAN_ERR_ARG, "buffer too small (%zu bytes needed)", s.size() + 1);
}

}  // extern "C"
