// noalloc.cu -- conan_deposit_static: the FP32 CIC deposit that allocates no
// device memory.
//
// The Lagrangian deposit of conan_pm sums the particles' corner weights into
// a 64-bit integer accumulator mesh that the handle allocates at creation.
// Some callers cannot allocate that mesh, nor anything else, at the point
// where they need a density:
//   * code inside a framework that has already reserved the device memory
//     for its own caching allocator (a cudaMalloc there fails, or fragments
//     the pool the framework manages);
//   * processes with a fixed device-memory budget negotiated up front, where
//     every buffer is accounted for before the work starts;
//   * loops with hard latency targets, where cudaMalloc / cudaFree would
//     serialise with the whole device.
// For them this entry point keeps the accumulator in one file-scope device
// array of fixed size (STATIC_CELLS cells, 16 MiB), which every GPU that loads
// the library holds until the process exits. The caller passes device
// pointers to the inputs and the output and nothing is allocated per call.
//
// Sharing rules: every call on a device uses the same array, so calls whose
// GPU work overlaps in time (different streams, or different host threads
// without ordering) race and give wrong densities; order them on one stream
// or with events. The array keeps the last call's contents, so each call
// clears the cells it uses before depositing (one memset); the clear comes
// first rather than last so that a call never depends on an earlier call
// having run to the end.
//
// Window choice, as the conan_pm handle makes it: the largest lattice tile
// whose shared-memory window fits and holds at most
// LAG_WINDOW_CELLS_PER_PARTICLE window cells per particle; otherwise (fine
// meshes, e.g. 32^3 particles on a 128^3 mesh) the largest tile with a
// two-cell window, i.e. every corner goes to the accumulator with one
// integer atomic. Both give the same integers.
#include <mutex>

#include "pm_kernels.cuh"

namespace conan {
namespace {

// Largest force mesh of conan_deposit_static: 2^21 cells (128^3, 2048^2,
// 2^21 in 1D), 8 bytes per cell.
constexpr size_t STATIC_CELLS = (size_t)CONAN_DEPOSIT_STATIC_MAX_CELLS;

// The accumulator. In host code this name is only a handle for
// cudaGetSymbolAddress, not a device address.
static __device__ __align__(256) unsigned long long g_static_acc[STATIC_CELLS];

// Per-device set-up: the array's device address, looked up with the device
// current, and the shared-memory limits of the kernels below.
struct DevSetup {
    bool done = false;
    unsigned long long *acc = nullptr;
};
constexpr int MAX_DEVICES = 64;
DevSetup g_setup[MAX_DEVICES];
std::mutex g_setup_mu;

template <int R, int LX, int LY, int LZ, int THREADS>
__global__ void __launch_bounds__(THREADS)
    k_deposit_static(Parts<float> P, Mesh m, LagWin win, unsigned long long *__restrict__ acc) {
    lag_tile<R, LX, LY, LZ, THREADS, false>(P, m, win, acc, nullptr, GKD{});
}

// Density contrast from the accumulator (units of 2^-23 particle weights,
// times the particle mass).
__global__ void __launch_bounds__(256) k_static_mesh(const unsigned long long *__restrict__ acc,
                                                     float *__restrict__ out, size_t n, double scale) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = (float)((double)acc[i] * (0x1p-23 * scale) - 1.0);
}

// Window of lattice tile V on an n^R lattice with f force cells per spacing:
// 1 and the window when the tile fits the lattice and its window fits
// shared memory, else 0. direct: a two-cell window (corners go to the
// accumulator directly).
template <int R, int V> int window_of(int n, int f, bool direct, LagWin *w, size_t *smem) {
    typedef LagTile<R, V> L;
    if (n < L::LX || (R >= 2 && n < L::LY) || (R == 3 && n < L::LZ)) return 0;
    LagWin x{};
    x.w[0] = direct ? 2 : L::LX * f + L::M;
    x.w[1] = R >= 2 ? (direct ? 2 : L::LY * f + L::M) : 1;
    x.w[2] = R == 3 ? (direct ? 2 : L::LZ * f + L::M) : 1;
    x.cells = (x.w[0] * x.w[1] * x.w[2] + 3) & ~3;
    size_t sh = (size_t)x.cells * LAG_PLANES * sizeof(uint32_t);
    if (sh > 112 * 1024) return 0;
    *w = x;
    *smem = sh;
    return 1;
}

template <int R, int V> constexpr double tile_particles() {
    return (double)LagTile<R, V>::LX * LagTile<R, V>::LY * LagTile<R, V>::LZ;
}

// The tile variant and window for an n^R lattice on an (f n)^R mesh, as the
// handle chooses them; -1 when the lattice is smaller than every tile.
template <int R> int choose_window(int n, int f, LagWin *w, size_t *smem) {
    int v = window_of<R, 0>(n, f, false, w, smem) ? 0 : window_of<R, 1>(n, f, false, w, smem) ? 1
            : window_of<R, 2>(n, f, false, w, smem) ? 2 : -1;
    const double per = v == 0 ? tile_particles<R, 0>() : v == 1 ? tile_particles<R, 1>() : tile_particles<R, 2>();
    if (v < 0 || (double)w->cells > LAG_WINDOW_CELLS_PER_PARTICLE * per)
        v = window_of<R, 0>(n, f, true, w, smem) ? 0 : window_of<R, 1>(n, f, true, w, smem) ? 1
            : window_of<R, 2>(n, f, true, w, smem) ? 2 : -1;
    return v;
}

template <int R, int V> int raise_smem_limit() {
    typedef LagTile<R, V> L;
    CONAN_CUDA(cudaFuncSetAttribute(k_deposit_static<R, L::LX, L::LY, L::LZ, L::THREADS>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, 112 * 1024));
    return CONAN_OK;
}

int setup_device(unsigned long long **acc) {
    int dev = 0;
    CONAN_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) return set_error(CONAN_ERR_UNSUPPORTED, "device %d: at most %d devices", dev, MAX_DEVICES);
    std::lock_guard<std::mutex> lock(g_setup_mu);
    DevSetup &s = g_setup[dev];
    if (!s.done) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_acc);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return set_error(CONAN_ERR_CUDA, "cudaGetSymbolAddress of the static accumulator failed: %s",
                             cudaGetErrorString(e));
        }
        CONAN_TRY((raise_smem_limit<1, 0>()));
        CONAN_TRY((raise_smem_limit<1, 1>()));
        CONAN_TRY((raise_smem_limit<1, 2>()));
        CONAN_TRY((raise_smem_limit<2, 0>()));
        CONAN_TRY((raise_smem_limit<2, 1>()));
        CONAN_TRY((raise_smem_limit<2, 2>()));
        CONAN_TRY((raise_smem_limit<3, 0>()));
        CONAN_TRY((raise_smem_limit<3, 1>()));
        CONAN_TRY((raise_smem_limit<3, 2>()));
        s.acc = (unsigned long long *)p;
        s.done = true;
    }
    *acc = s.acc;
    return CONAN_OK;
}

template <int R, int V>
int launch(const Parts<float> &P, const Mesh &m, const LagWin &w, size_t smem, unsigned long long *acc,
           cudaStream_t st) {
    typedef LagTile<R, V> L;
    const int n = 1 << P.mshift;
    const unsigned tiles = (unsigned)((n / L::LX) * (R >= 2 ? n / L::LY : 1) * (R == 3 ? n / L::LZ : 1));
    k_deposit_static<R, L::LX, L::LY, L::LZ, L::THREADS><<<tiles, L::THREADS, smem, st>>>(P, m, w, acc);
    CONAN_LAUNCHED();
    return CONAN_OK;
}

template <int R>
int deposit_static(int n, int f, const float *const *d, float *out, cudaStream_t st) {
    LagWin w{};
    size_t smem = 0;
    const int v = choose_window<R>(n, f, &w, &smem);
    if (v < 0)
        return set_error(CONAN_ERR_UNSUPPORTED,
                         "conan_deposit_static: %d particles per side is below the smallest lattice tile (%d) "
                         "in %d dimensions",
                         n, LagTile<R, 2>::LX, R);
    unsigned long long *acc = nullptr;
    CONAN_TRY(setup_device(&acc));
    const Mesh m = make_mesh(R, n * f, 1);
    Parts<float> P{};
    for (int k = 0; k < R; ++k) P.d[k] = const_cast<float *>(d[k]);
    P.np = (size_t)1 << (R * ilog2(n));
    P.mshift = ilog2(n);
    P.f = f;
    P.bshift = R * P.mshift;
    CONAN_CUDA(cudaMemsetAsync(acc, 0, m.cells * sizeof(unsigned long long), st));
    if (v == 0) CONAN_TRY((launch<R, 0>(P, m, w, smem, acc, st)));
    if (v == 1) CONAN_TRY((launch<R, 1>(P, m, w, smem, acc, st)));
    if (v == 2) CONAN_TRY((launch<R, 2>(P, m, w, smem, acc, st)));
    const double mass = (double)((size_t)1 << (R * ilog2(f)));
    k_static_mesh<<<(unsigned)((m.cells + 255) / 256), 256, 0, st>>>(acc, out, m.cells, mass);
    CONAN_LAUNCHED();
    return CONAN_OK;
}

}  // namespace
}  // namespace conan

using namespace conan;

extern "C" int conan_deposit_static(int dim, int n_mass, int f, const float *d0, const float *d1, const float *d2,
                                    float *delta_out, void *stream) {
    if (dim < 1 || dim > 3) return set_error(CONAN_ERR_UNSUPPORTED, "conan_deposit_static: dim = %d (1..3)", dim);
    if (n_mass < 2 || !is_pow2(n_mass) || f < 1 || !is_pow2(f))
        return set_error(CONAN_ERR_ARG, "conan_deposit_static: n_mass = %d and f = %d must be powers of two",
                         n_mass, f);
    const long long nf = (long long)n_mass * f;
    long long cells = 1;
    for (int k = 0; k < dim; ++k) {
        cells *= nf;
        if (cells > (long long)STATIC_CELLS)
            return set_error(CONAN_ERR_ARG,
                             "conan_deposit_static: a force mesh of %lld^%d cells exceeds the static accumulator "
                             "(at most %zu cells); use conan_pm_density",
                             nf, dim, STATIC_CELLS);
    }
    const float *d[3] = {d0, d1, d2};
    for (int k = 0; k < dim; ++k)
        if (!d[k]) return set_error(CONAN_ERR_ARG, "conan_deposit_static: null displacement array %d", k);
    if (!delta_out) return set_error(CONAN_ERR_ARG, "conan_deposit_static: null output");
    cudaStream_t st = (cudaStream_t)stream;
    switch (dim) {
        case 1: return deposit_static<1>(n_mass, f, d, delta_out, st);
        case 2: return deposit_static<2>(n_mass, f, d, delta_out, st);
        default: return deposit_static<3>(n_mass, f, d, delta_out, st);
    }
}
