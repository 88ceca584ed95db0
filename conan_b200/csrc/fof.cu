// fof.cu -- the `fof` tool on the GPU: friends-of-friends groups of a
// snapshot's particles, fof_run<R> (src/fof/fof.cc:164-279).
//
// The reference links two particles when the squared length of their raw
// coordinate difference, wrapped once per axis into [-L/2, L/2] (Proximity,
// src/fof/fof.cc:71-99), is at most the squared linking length, and numbers
// the connected groups from 1 in the order of their lowest particle index
// (the flood fill started from every untagged particle in index order,
// src/fof/fof.cc:183-231). The result is a partition plus that numbering, so
// any order of discovery gives the same tags. Here:
//   bin      every particle's cell on a grid whose cells are no smaller than
//            the linking length (wrapped coordinates) and its rank in the
//            cell from an integer counter;
//   scan     cell offsets;
//   scatter  particle indices and coordinates (one array per axis) in cell
//            order;
//   link     one thread per sorted particle tests the particles after it in
//            its own cell and all particles of the (3^R - 1) / 2 neighbour
//            cells that lie ahead of its cell, so every pair within reach is
//            tested exactly once, in FP64 with the reference's operation order
//            and no fused multiply-add; a linked pair joins two trees of a
//            lock-free union-find that always hooks the larger root under the
//            smaller one, so every root is the lowest index of its tree;
//   roots    every particle's root (a read-only walk once the links are in);
//   number   exclusive scan of the root flags = group number - 1.
#include <algorithm>
#include <cmath>

#include "pm.cuh"
#include "scan.cuh"

namespace conan {
namespace {

constexpr int FOF_T = 256;
constexpr int FOF_UNITE_LIMIT = 1 << 24;  // retries of one union (each one is another thread's hook)

struct FofGrid {
    int nc;        // cells per side (1 or >= 3)
    double L;      // box size
    double half;   // L / 2
    double inv_h;  // nc / L
    double rsqr;   // linking length squared
};

// Cell of a position: the coordinate wrapped into [0, L), nc cells per side.
// Explicitly rounded operations, so that the binning and the link kernel
// (which recomputes it) agree bit for bit.
template <int R>
__device__ inline uint32_t fof_cell(const double *x, const FofGrid &g, int *c) {
    uint32_t id = 0;
#pragma unroll
    for (int k = R - 1; k >= 0; --k) {
        const double w = __dsub_rn(x[k], __dmul_rn(floor(__ddiv_rn(x[k], g.L)), g.L));
        int ck = (int)__dmul_rn(w, g.inv_h);
        ck = ck < 0 ? 0 : (ck >= g.nc ? g.nc - 1 : ck);
        c[k] = ck;
        id = id * (uint32_t)g.nc + (uint32_t)ck;
    }
    return id;
}

// Proximity::operator()(size_t), src/fof/fof.cc:85-99: b = x_j - x_i, one
// wrap per axis, d.sqr() summed in axis order, compared with r * r.
template <int R>
__device__ inline bool fof_linked(const double *a, const double *b, const FofGrid &g) {
    double v = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const double e = __dsub_rn(b[k], a[k]);
        const double d = e > g.half ? __dsub_rn(e, g.L) : (e < -g.half ? __dadd_rn(e, g.L) : e);
        v = __dadd_rn(v, __dmul_rn(d, d));
    }
    return v <= g.rsqr;
}

// Root of x with path halving. Parents always point to lower indices, so the
// walk ends; a halving store writes an ancestor of x, which stays valid
// whatever other threads do to the tree meanwhile. Loads bypass L1 so that
// hooks made by other SMs are seen.
__device__ inline uint32_t fof_find(uint32_t *par, uint32_t x) {
    for (;;) {
        const uint32_t p = __ldcg(par + x);
        if (p == x) return x;
        const uint32_t g = __ldcg(par + p);
        if (g == p) return p;
        __stcg(par + x, g);
        x = g;
    }
}

// Joins the trees of a and b: the larger root is hooked under the smaller
// one with a compare-and-swap that only succeeds while it is still a root.
__device__ inline bool fof_unite(uint32_t *par, uint32_t a, uint32_t b) {
    for (int it = 0; it < FOF_UNITE_LIMIT; ++it) {
        a = fof_find(par, a);
        b = fof_find(par, b);
        if (a == b) return true;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        const uint32_t old = atomicCAS(par + a, a, b);
        if (old == a) return true;
        a = old;  // hooked by another thread meanwhile: continue from there
    }
    return false;
}

template <int R>
__global__ void __launch_bounds__(FOF_T) k_fof_bin(const double *__restrict__ X, size_t n, FofGrid g,
                                                   uint32_t *__restrict__ cell, uint32_t *__restrict__ slot,
                                                   uint32_t *__restrict__ count) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i >= n) return;
    double x[3];
    int c[3];
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = X[i * R + k];
    const uint32_t id = fof_cell<R>(x, g, c);
    cell[i] = id;
    slot[i] = atomicAdd(count + id, 1u);
}

template <int R>
__global__ void __launch_bounds__(FOF_T) k_fof_scatter(const double *__restrict__ X, size_t n,
                                                       const uint32_t *__restrict__ cell,
                                                       const uint32_t *__restrict__ slot,
                                                       const uint32_t *__restrict__ off,
                                                       uint32_t *__restrict__ order, double *__restrict__ S,
                                                       uint32_t *__restrict__ par) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i >= n) return;
    const size_t t = (size_t)off[cell[i]] + slot[i];
    order[t] = (uint32_t)i;
#pragma unroll
    for (int k = 0; k < R; ++k) S[(size_t)k * n + t] = X[i * R + k];
    par[i] = (uint32_t)i;
}

// Tests sorted particle t against the particles u in [u0, u1) of one cell.
template <int R>
__device__ inline void fof_test_range(const double *xi, uint32_t i, size_t u0, size_t u1, size_t n,
                                      const double *__restrict__ S, const uint32_t *__restrict__ order,
                                      const FofGrid &g, uint32_t *par, int *err) {
    for (size_t u = u0; u < u1; ++u) {
        double xj[3];
#pragma unroll
        for (int k = 0; k < R; ++k) xj[k] = __ldg(S + (size_t)k * n + u);
        if (fof_linked<R>(xi, xj, g) && !fof_unite(par, i, __ldg(order + u))) atomicOr(err, 1);
    }
}

template <int R>
__global__ void __launch_bounds__(FOF_T) k_fof_link(const double *__restrict__ S,
                                                    const uint32_t *__restrict__ order,
                                                    const uint32_t *__restrict__ off, size_t n, FofGrid g,
                                                    uint32_t *par, int *err) {
    const size_t t = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (t >= n) return;
    double xi[3];
    int c[3];
#pragma unroll
    for (int k = 0; k < R; ++k) xi[k] = S[(size_t)k * n + t];
    const uint32_t i = order[t];
    const uint32_t own = fof_cell<R>(xi, g, c);
    fof_test_range<R>(xi, i, t + 1, off[own + 1], n, S, order, g, par, err);
    if (g.nc == 1) return;
    // the neighbour offsets o in {-1,0,1}^R whose last non-zero component
    // (highest axis first) is +1: half of the 3^R - 1 neighbours
    constexpr int NB = (R == 2 ? 9 : 27);
    for (int q = NB / 2 + 1; q < NB; ++q) {
        int o[3] = {q % 3 - 1, (q / 3) % 3 - 1, q / 9 - 1};
        uint32_t id = 0;
#pragma unroll
        for (int k = R - 1; k >= 0; --k) {
            int ck = c[k] + o[k];
            ck = ck < 0 ? ck + g.nc : (ck >= g.nc ? ck - g.nc : ck);
            id = id * (uint32_t)g.nc + (uint32_t)ck;
        }
        fof_test_range<R>(xi, i, off[id], off[id + 1], n, S, order, g, par, err);
    }
}

// Every particle's root into a separate array, flag = 1 for roots. The walk
// only reads the parents: a path-halving store in this pass could overwrite
// a root another thread has just written with an older ancestor.
__global__ void __launch_bounds__(FOF_T) k_fof_roots(const uint32_t *__restrict__ par, size_t n,
                                                     uint32_t *__restrict__ root, uint32_t *__restrict__ flag) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i >= n) return;
    uint32_t r = (uint32_t)i, p = par[r];
    while (p != r) {
        r = p;
        p = par[r];
    }
    root[i] = r;
    flag[i] = r == (uint32_t)i ? 1u : 0u;
}

__global__ void __launch_bounds__(FOF_T) k_fof_tags(const uint32_t *__restrict__ root,
                                                    const uint32_t *__restrict__ gnum, size_t n,
                                                    unsigned long long *__restrict__ tags) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i >= n) return;
    tags[i] = (unsigned long long)gnum[root[i]] + 1ull;
}

inline unsigned blocks(size_t n) { return (unsigned)((n + FOF_T - 1) / FOF_T); }

}  // namespace

// Grid and device buffers of one problem size; reused across runs.
struct FofEngine {
    int R = 3, device = 0;
    size_t n = 0, cells = 0;
    FofGrid g{};
    cudaStream_t st = nullptr;
    double *X = nullptr, *S = nullptr;
    uint32_t *cell = nullptr, *slot = nullptr, *order = nullptr, *par = nullptr, *count = nullptr,
             *off = nullptr, *bsum = nullptr;
    unsigned long long *tags = nullptr;
    uint32_t *ngroups_h = nullptr;  // pinned
    int *err = nullptr;

    ~FofEngine() {
        if (st) cudaStreamSynchronize(st);
        cudaFree(X);
        cudaFree(S);
        cudaFree(cell);
        cudaFree(slot);
        cudaFree(order);
        cudaFree(par);
        cudaFree(count);
        cudaFree(off);
        cudaFree(bsum);
        cudaFree(tags);
        cudaFree(err);
        cudaFreeHost(ngroups_h);
        if (st) cudaStreamDestroy(st);
    }

    int init(const conan_fof_params &p) {
        R = p.dim;
        device = p.device;
        n = (size_t)p.n_particles;
        // cells no smaller than the linking length (with a margin far above
        // the rounding of the wrap), at most about one per particle
        double q = p.size / (p.linking_length * (1.0 + 1e-9));
        long long nc = q >= 2147483647.0 ? 2147483647LL : (long long)q;
        long long cap = 1;
        while (true) {
            long long c1 = cap + 1, v = 1;
            for (int k = 0; k < R; ++k) v *= c1;
            if (v > (long long)std::max<size_t>(n, 27) || v > (1LL << 30)) break;
            cap = c1;
        }
        nc = std::min(nc, cap);
        if (nc < 3) nc = 1;
        g.nc = (int)nc;
        g.L = p.size;
        g.half = p.size / 2;
        g.inv_h = (double)nc / p.size;
        g.rsqr = p.linking_length * p.linking_length;
        cells = 1;
        for (int k = 0; k < R; ++k) cells *= (size_t)nc;
        const size_t nb = (std::max(cells, n) + SCAN_CHUNK - 1) / SCAN_CHUNK;
        CONAN_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CONAN_CUDA(cudaMalloc(&X, n * R * sizeof(double)));
        CONAN_CUDA(cudaMalloc(&S, n * R * sizeof(double)));
        CONAN_CUDA(cudaMalloc(&cell, (n + 1) * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&slot, n * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&order, n * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&par, n * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&count, cells * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&off, (cells + 1) * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&bsum, nb * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&tags, n * sizeof(unsigned long long)));
        CONAN_CUDA(cudaMalloc(&err, sizeof(int)));
        CONAN_CUDA(cudaMallocHost(&ngroups_h, 2 * sizeof(uint32_t)));
        CONAN_CUDA(cudaMemsetAsync(count, 0, cells * sizeof(uint32_t), st));
        CONAN_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }

    void scan(uint32_t *cnt, size_t m, uint32_t *out, cudaStream_t s) {
        const size_t nb = (m + SCAN_CHUNK - 1) / SCAN_CHUNK;
        k_scan_partial<<<(unsigned)nb, SCAN_T, 0, s>>>(cnt, m, bsum);
        k_scan_blocks<<<1, 1024, 0, s>>>(bsum, (int)nb);
        k_scan_final<<<(unsigned)nb, SCAN_T, 0, s>>>(cnt, m, bsum, out);
    }

    // Groups of the positions in Xd (device, n x R doubles); tags into tg
    // (device, n values). Enqueued on `s`; the group count is read back.
    template <int RR> int run_t(const double *Xd, unsigned long long *tg, cudaStream_t s, uint64_t *ngroups) {
        k_fof_bin<RR><<<blocks(n), FOF_T, 0, s>>>(Xd, n, g, cell, slot, count);
        scan(count, cells, off, s);
        k_fof_scatter<RR><<<blocks(n), FOF_T, 0, s>>>(Xd, n, cell, slot, off, order, S, par);
        k_fof_link<RR><<<blocks(n), FOF_T, 0, s>>>(S, order, off, n, g, par, err);
        // roots into `order` and root flags into `slot` (both free after the
        // link), group numbers into `cell`
        k_fof_roots<<<blocks(n), FOF_T, 0, s>>>(par, n, order, slot);
        scan(slot, n, cell, s);
        k_fof_tags<<<blocks(n), FOF_T, 0, s>>>(order, cell, n, tg);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return set_error(CONAN_ERR_CUDA, "fof kernel launch failed: %s", cudaGetErrorString(e));
        int herr = 0;
        CONAN_CUDA(cudaMemcpyAsync(ngroups_h, cell + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CONAN_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        CONAN_CUDA(cudaMemsetAsync(err, 0, sizeof(int), s));
        CONAN_CUDA(cudaStreamSynchronize(s));
        if (herr)
            return set_error(CONAN_ERR_STATE, "fof: a union did not finish within %d retries", FOF_UNITE_LIMIT);
        if (ngroups) *ngroups = ngroups_h[0];
        return CONAN_OK;
    }

    int run_device(const double *Xd, unsigned long long *tg, cudaStream_t s, uint64_t *ngroups) {
        return R == 2 ? run_t<2>(Xd, tg, s, ngroups) : run_t<3>(Xd, tg, s, ngroups);
    }

    int run_host(const double *Xh, unsigned long long *tg_h, uint64_t *ngroups) {
        CONAN_CUDA(cudaMemcpyAsync(X, Xh, n * R * sizeof(double), cudaMemcpyHostToDevice, st));
        CONAN_TRY(run_device(X, tags, st, ngroups));
        CONAN_CUDA(cudaMemcpyAsync(tg_h, tags, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        CONAN_CUDA(cudaStreamSynchronize(st));
        return CONAN_OK;
    }
};

int check_fof_params(const conan_fof_params *p) {
    if (!p) return set_error(CONAN_ERR_ARG, "null parameters");
    if (p->dim != 2 && p->dim != 3) return set_error(CONAN_ERR_UNSUPPORTED, "fof: dim = %d (2 or 3)", p->dim);
    if (p->n_particles < 1 || p->n_particles >= (1ULL << 32) - 1)
        return set_error(CONAN_ERR_ARG, "fof: particle count %llu outside 1 .. 2^32 - 2", p->n_particles);
    if (!(p->size > 0) || !std::isfinite(p->size)) return set_error(CONAN_ERR_ARG, "fof: box size must be positive");
    if (!(p->linking_length > 0) || !std::isfinite(p->linking_length))
        return set_error(CONAN_ERR_ARG, "fof: linking length must be positive");
    return CONAN_OK;
}

}  // namespace conan

using namespace conan;

struct conan_fof_engine {
    FofEngine e;
};

extern "C" conan_fof_engine *conan_fof_create(const conan_fof_params *p) {
    if (check_fof_params(p) != CONAN_OK) return nullptr;
    if (device_guard(p->device) != CONAN_OK) return nullptr;
    conan_fof_engine *h = new conan_fof_engine;
    if (h->e.init(*p) != CONAN_OK) {
        std::string msg = last_error();
        delete h;
        set_error(CONAN_ERR_ALLOC, "%s", msg.c_str());
        return nullptr;
    }
    return h;
}

extern "C" void conan_fof_destroy(conan_fof_engine *h) {
    if (!h) return;
    cudaSetDevice(h->e.device);
    delete h;
}

extern "C" int conan_fof_run(conan_fof_engine *h, const double *X, unsigned long long *tags, unsigned long long *n_groups) {
    if (!h) return set_error(CONAN_ERR_ARG, "null fof handle");
    if (!X || !tags) return set_error(CONAN_ERR_ARG, "fof: null positions or tags");
    CONAN_TRY(device_guard(h->e.device));
    uint64_t ng = 0;
    CONAN_TRY(h->e.run_host(X, tags, &ng));
    if (n_groups) *n_groups = ng;
    return CONAN_OK;
}

extern "C" int conan_fof_run_device(conan_fof_engine *h, const double *X, unsigned long long *tags,
                                    unsigned long long *n_groups, void *stream) {
    if (!h) return set_error(CONAN_ERR_ARG, "null fof handle");
    if (!X || !tags) return set_error(CONAN_ERR_ARG, "fof: null positions or tags");
    CONAN_TRY(device_guard(h->e.device));
    uint64_t ng = 0;
    CONAN_TRY(h->e.run_device(X, tags, (cudaStream_t)stream, &ng));
    if (n_groups) *n_groups = ng;
    return CONAN_OK;
}

extern "C" int conan_fof(const conan_fof_params *p, const double *X, unsigned long long *tags,
                         unsigned long long *n_groups) {
    CONAN_TRY(check_fof_params(p));
    if (!X || !tags) return set_error(CONAN_ERR_ARG, "fof: null positions or tags");
    conan_fof_engine *h = conan_fof_create(p);
    if (!h) return CONAN_ERR_ALLOC;
    int rc = conan_fof_run(h, X, tags, n_groups);
    conan_fof_destroy(h);
    return rc;
}
