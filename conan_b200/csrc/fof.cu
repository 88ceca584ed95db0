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
//   keys     every particle's row -- its cell in the transverse axes (y, or
//            y and z) on a grid of cells no smaller than the linking length,
//            wrapped coordinates -- and its wrapped x quantised to 2^16
//            steps, as one 64-bit key; an integer count per row;
//   sort     counting sort by row (offsets from the counts), then every row
//            sorted by (x, particle index): across the lanes of a warp up to
//            32 particles, in shared memory up to 4096; a longer row sends
//            the whole array through a stable radix sort of (key, particle
//            index) instead (radix.cuh). Either way: rows in order, x
//            ascending inside a row, ties in particle order;
//   gather   coordinates (one array per axis) in sorted order;
//   link     one thread per sorted particle tests, in its own row, the
//            particles ahead of it in cyclic x order within the linking
//            length, and in the forward half of the neighbouring rows
//            ((3^(R-1) - 1) / 2 rows) those within the linking length in x,
//            found by binary search; every pair within reach is tested
//            exactly once, in FP64 with the reference's operation order and
//            no fused multiply-add. A linked pair joins two trees of a
//            lock-free union-find that always hooks the larger root under the
//            smaller one, so every root is the lowest index of its tree;
//   roots    every particle's root (a read-only walk once the links are in);
//   number   exclusive scan of the root flags = group number - 1.
// Against cubic cells, the row-and-window search tests candidates from a
// volume of 2 ll x (3 ll)^(R-1) around each particle instead of (3 h)^R with
// cells h >= ll; inside halos that is most of the work.
#include <algorithm>
#include <cmath>

#include "pm.cuh"
#include "radix.cuh"
#include "scan.cuh"

namespace conan {
namespace {

constexpr int FOF_T = 256;
constexpr int FOF_UNITE_LIMIT = 1 << 24;  // retries of one union (each one is another thread's hook)
constexpr int FOF_XB = 16;                 // bits of the quantised x in the sort key
constexpr uint32_t FOF_XN = 1u << FOF_XB;
constexpr uint64_t FOF_XMASK = FOF_XN - 1;
constexpr uint32_t FOF_NONE = 0xffffffffu;

struct FofGrid {
    int nr;         // row cells per transverse axis (1 or >= 3)
    int wq;         // x window in quanta; whole rows when 2 wq + 1 >= 2^16
    double L;       // box size
    double half;    // L / 2
    double inv_h;   // nr / L
    double xscale;  // 2^16 / L
    double rsqr;    // linking length squared
};

// Wrapped coordinate in [0, L], explicitly rounded.
__device__ inline double fof_wrap(double x, const FofGrid &g) {
    return __dsub_rn(x, __dmul_rn(floor(__ddiv_rn(x, g.L)), g.L));
}

// Row of a position (transverse cells, highest axis most significant) and
// its key: row << 16 | quantised x.
template <int R>
__device__ inline uint64_t fof_key(const double *x, const FofGrid &g, uint32_t *row_out) {
    uint32_t row = 0;
#pragma unroll
    for (int k = R - 1; k >= 1; --k) {
        int ck = (int)__dmul_rn(fof_wrap(x[k], g), g.inv_h);
        ck = ck < 0 ? 0 : (ck >= g.nr ? g.nr - 1 : ck);
        row = row * (uint32_t)g.nr + (uint32_t)ck;
    }
    long long q = (long long)__dmul_rn(fof_wrap(x[0], g), g.xscale);
    q = q < 0 ? 0 : (q >= (long long)FOF_XN ? (long long)FOF_XN - 1 : q);
    *row_out = row;
    return ((uint64_t)row << FOF_XB) | (uint64_t)q;
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
// Returns the root of the joined tree as this thread last saw it (a cheap
// starting point for the next union of the same particle), FOF_NONE if it
// gave up.
__device__ inline uint32_t fof_unite(uint32_t *par, uint32_t a, uint32_t b) {
    for (int it = 0; it < FOF_UNITE_LIMIT; ++it) {
        a = fof_find(par, a);
        b = fof_find(par, b);
        if (a == b) return a;
        const uint32_t hi = a > b ? a : b, lo = a > b ? b : a;
        const uint32_t old = atomicCAS(par + hi, hi, lo);
        if (old == hi) return lo;
        a = old;  // hi was hooked by another thread meanwhile: continue from there
        b = lo;
    }
    return FOF_NONE;
}

// Key of every particle (particle order) and its rank in its row from an
// integer counter.
template <int R>
__global__ void __launch_bounds__(FOF_T) k_fof_keys(const double *__restrict__ X, size_t n, FofGrid g,
                                                    uint64_t *__restrict__ keys, uint32_t *__restrict__ slot,
                                                    uint32_t *__restrict__ rowcount) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i >= n) return;
    double x[3];
#pragma unroll
    for (int k = 0; k < R; ++k) x[k] = X[i * R + k];
    uint32_t row;
    keys[i] = fof_key<R>(x, g, &row);
    slot[i] = atomicAdd(rowcount + row, 1u);
}

// Counting sort by row: every particle at its row's offset plus its rank
// (the order inside a row is put right by the row sorts).
__global__ void __launch_bounds__(FOF_T) k_fof_place(const uint64_t *__restrict__ kp, const uint32_t *__restrict__ slot,
                                                     const uint32_t *__restrict__ rowoff, size_t n,
                                                     uint64_t *__restrict__ keys, uint32_t *__restrict__ order) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i >= n) return;
    const uint64_t key = kp[i];
    const size_t t = (size_t)rowoff[key >> FOF_XB] + slot[i];
    keys[t] = key;
    order[t] = (uint32_t)i;
}

constexpr int FOF_BIG = 4096;  // longest row sorted in shared memory

// Sort value of a sorted slot: quantised x above the particle index (unique,
// and the order a stable sort by key from particle order would give).
__device__ inline uint64_t fof_sortval(const uint64_t *keys, const uint32_t *order, size_t t) {
    return ((keys[t] & FOF_XMASK) << 32) | order[t];
}

// One warp per row: rows of up to 32 particles are sorted by (x, index) with
// a bitonic network across the lanes; longer rows are queued for
// k_fof_rowsort_big (up to FOF_BIG) or flagged in nbig[1] (longer).
__global__ void __launch_bounds__(256) k_fof_rowsort_small(uint64_t *__restrict__ keys, uint32_t *__restrict__ order,
                                                           const uint32_t *__restrict__ rowoff, size_t rows,
                                                           uint32_t *__restrict__ big, uint32_t *__restrict__ nbig) {
    const int lane = threadIdx.x & 31;
    const size_t nw = (size_t)gridDim.x * (256 / 32);
    for (size_t r = ((size_t)blockIdx.x * 256 + threadIdx.x) >> 5; r < rows; r += nw) {
        const size_t rs = rowoff[r];
        const uint32_t m = rowoff[r + 1] - (uint32_t)rs;
        if (m <= 1) continue;
        if (m > 32) {
            if (lane == 0) {
                if (m > (uint32_t)FOF_BIG) atomicOr(nbig + 1, 1u);
                else big[atomicAdd(nbig, 1u)] = (uint32_t)r;
            }
            continue;
        }
        uint64_t v = (uint32_t)lane < m ? fof_sortval(keys, order, rs + lane) : ~0ull;
#pragma unroll
        for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
            for (int j = k >> 1; j > 0; j >>= 1) {
                const uint64_t o = __shfl_xor_sync(FULL, v, j);
                const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
                v = keep_min ? (v < o ? v : o) : (v > o ? v : o);
            }
        }
        if ((uint32_t)lane < m) {
            keys[rs + lane] = ((uint64_t)r << FOF_XB) | (v >> 32);
            order[rs + lane] = (uint32_t)v;
        }
    }
}

// One CTA per queued row (33 .. FOF_BIG particles): bitonic sort in shared
// memory over the next power of two, padded with the largest value.
__global__ void __launch_bounds__(256) k_fof_rowsort_big(uint64_t *__restrict__ keys, uint32_t *__restrict__ order,
                                                         const uint32_t *__restrict__ rowoff,
                                                         const uint32_t *__restrict__ big,
                                                         const uint32_t *__restrict__ nbig) {
    __shared__ uint64_t sv[FOF_BIG];
    const uint32_t nq = nbig[0];
    for (uint32_t b = blockIdx.x; b < nq; b += gridDim.x) {
        const uint32_t r = big[b];
        const size_t rs = rowoff[r];
        const uint32_t m = rowoff[r + 1] - (uint32_t)rs;
        uint32_t P = 64;
        while (P < m) P <<= 1;
        for (uint32_t j = threadIdx.x; j < P; j += 256) sv[j] = j < m ? fof_sortval(keys, order, rs + j) : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t x = threadIdx.x; x < P; x += 256) {
                    const uint32_t y = x ^ j;
                    if (y > x) {
                        const uint64_t a = sv[x], c = sv[y];
                        if ((a > c) == ((x & k) == 0)) {
                            sv[x] = c;
                            sv[y] = a;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t j = threadIdx.x; j < m; j += 256) {
            const uint64_t v = sv[j];
            keys[rs + j] = ((uint64_t)r << FOF_XB) | (v >> 32);
            order[rs + j] = (uint32_t)v;
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(FOF_T) k_fof_iota(uint32_t *__restrict__ v, size_t n) {
    const size_t i = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (i < n) v[i] = (uint32_t)i;
}

template <int R>
__global__ void __launch_bounds__(FOF_T) k_fof_gather(const double *__restrict__ X, size_t n,
                                                      const uint32_t *__restrict__ order, double *__restrict__ S,
                                                      uint32_t *__restrict__ par) {
    const size_t t = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (t >= n) return;
    const uint32_t i = order[t];
#pragma unroll
    for (int k = 0; k < R; ++k) S[(size_t)k * n + t] = X[(size_t)i * R + k];
    par[t] = (uint32_t)t;  // every particle its own parent (par is indexed by particle)
}

struct FofLink {
    const double *S;
    const uint64_t *keys;
    const uint32_t *order;
    const uint32_t *rowoff;
    size_t n;
    FofGrid g;
    uint32_t *par;
    int *err;
};

// Tests sorted particle t (coordinates xi, index i, last known root ri)
// against sorted particle u.
template <int R>
__device__ inline void fof_test(const FofLink &a, const double *xi, uint32_t i, uint32_t &ri, size_t u) {
    double xj[3];
#pragma unroll
    for (int k = 0; k < R; ++k) xj[k] = __ldg(a.S + (size_t)k * a.n + u);
    if (!fof_linked<R>(xi, xj, a.g)) return;
    ri = fof_unite(a.par, ri, __ldg(a.order + u));
    if (ri == FOF_NONE) {
        atomicOr(a.err, 1);
        ri = i;
    }
}

// Tests the particles of sorted range [u, end) whose quantised x is at most
// qmax (keys are sorted, so the run stops at the first larger one).
template <int R>
__device__ inline void fof_run_to(const FofLink &a, const double *xi, uint32_t i, uint32_t &ri, size_t u, size_t end,
                                  uint64_t kmax) {
    for (; u < end && __ldg(a.keys + u) <= kmax; ++u) fof_test<R>(a, xi, i, ri, u);
}

// First sorted position in [lo, hi) whose key is >= k.
__device__ inline size_t fof_lower(const uint64_t *keys, size_t lo, size_t hi, uint64_t k) {
    while (lo < hi) {
        const size_t mid = lo + ((hi - lo) >> 1);
        if (__ldg(keys + mid) < k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Tests the particles of row `row` whose quantised x lies in [qa, qb].
template <int R>
__device__ inline void fof_row_segment(const FofLink &a, const double *xi, uint32_t i, uint32_t &ri, size_t rs,
                                       size_t re, uint64_t rk, long long qa, long long qb) {
    const size_t u = fof_lower(a.keys, rs, re, rk | (uint64_t)qa);
    fof_run_to<R>(a, xi, i, ri, u, re, rk | (uint64_t)qb);
}

// The x window [xq - wq, xq + wq] (cyclic) of one neighbour row.
template <int R>
__device__ inline void fof_row_window(const FofLink &a, const double *xi, uint32_t i, uint32_t &ri, uint32_t row,
                                      long long xq, bool whole) {
    const size_t rs = a.rowoff[row], re = a.rowoff[row + 1];
    if (rs == re) return;
    const uint64_t rk = (uint64_t)row << FOF_XB;
    if (whole) {
        for (size_t u = rs; u < re; ++u) fof_test<R>(a, xi, i, ri, u);
        return;
    }
    const long long lo = xq - a.g.wq, hi = xq + a.g.wq, N = FOF_XN;
    if (lo < 0) {
        fof_row_segment<R>(a, xi, i, ri, rs, re, rk, lo + N, N - 1);
        fof_row_segment<R>(a, xi, i, ri, rs, re, rk, 0, hi);
    } else if (hi >= N) {
        fof_row_segment<R>(a, xi, i, ri, rs, re, rk, lo, N - 1);
        fof_row_segment<R>(a, xi, i, ri, rs, re, rk, 0, hi - N);
    } else {
        fof_row_segment<R>(a, xi, i, ri, rs, re, rk, lo, hi);
    }
}

template <int R>
__global__ void __launch_bounds__(FOF_T) k_fof_link(FofLink a) {
    const size_t t = (size_t)blockIdx.x * FOF_T + threadIdx.x;
    if (t >= a.n) return;
    double xi[3];
#pragma unroll
    for (int k = 0; k < R; ++k) xi[k] = a.S[(size_t)k * a.n + t];
    const uint32_t i = a.order[t];
    uint32_t ri = i;
    const uint64_t key = a.keys[t];
    const uint32_t row = (uint32_t)(key >> FOF_XB);
    const long long xq = (long long)(key & FOF_XMASK);
    const bool whole = 2 * (long long)a.g.wq + 1 >= (long long)FOF_XN;
    const size_t rs = a.rowoff[row], re = a.rowoff[row + 1];
    // own row: the particles ahead of t in cyclic x order, up to wq ahead
    if (whole) {
        for (size_t u = t + 1; u < re; ++u) fof_test<R>(a, xi, i, ri, u);
    } else {
        const uint64_t rk = (uint64_t)row << FOF_XB;
        const long long hi = xq + a.g.wq;
        fof_run_to<R>(a, xi, i, ri, t + 1, re, rk | (uint64_t)(hi < (long long)FOF_XN ? hi : (long long)FOF_XN - 1));
        if (hi >= (long long)FOF_XN) fof_run_to<R>(a, xi, i, ri, rs, t, rk | (uint64_t)(hi - FOF_XN));
    }
    if (a.g.nr == 1) return;
    // the forward half of the neighbouring rows: y + 1 (2D); (y+-1, z+1),
    // (y, z+1), (y+1, z) (3D)
    const int nr = a.g.nr;
    const int cy = (int)(row % (uint32_t)nr), cz = R == 3 ? (int)(row / (uint32_t)nr) : 0;
    constexpr int NF = R == 2 ? 1 : 4;
    const int dy[4] = {1, -1, 0, 1}, dz[4] = {0, 1, 1, 1};
#pragma unroll
    for (int f = 0; f < NF; ++f) {
        int y = cy + dy[f], z = cz + dz[f];
        y = y < 0 ? y + nr : (y >= nr ? y - nr : y);
        z = z >= nr ? z - nr : z;
        const uint32_t nrow = R == 2 ? (uint32_t)y : (uint32_t)z * (uint32_t)nr + (uint32_t)y;
        fof_row_window<R>(a, xi, i, ri, nrow, xq, whole);
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
    int R = 3, device = 0, key_bits = 0;
    size_t n = 0, rows = 0;
    FofGrid g{};
    cudaStream_t st = nullptr;
    double *X = nullptr, *S = nullptr;
    uint64_t *keys[2] = {nullptr, nullptr};
    uint32_t *vals[2] = {nullptr, nullptr};
    uint32_t *par = nullptr, *rowcount = nullptr, *rowoff = nullptr, *flag = nullptr, *gnum = nullptr,
             *bh = nullptr, *boff = nullptr, *bsum = nullptr, *bigrows = nullptr, *nbig = nullptr;
    unsigned long long *tags = nullptr;
    uint32_t *ngroups_h = nullptr, *nbig_h = nullptr;  // pinned
    int *err = nullptr;
    int sort_blocks = 0;
    bool used_radix = false;  // the last run's rows were too long for the row sorts

    ~FofEngine() {
        if (st) cudaStreamSynchronize(st);
        for (void *q : {(void *)X, (void *)S, (void *)keys[0], (void *)keys[1], (void *)vals[0], (void *)vals[1],
                        (void *)par, (void *)rowcount, (void *)rowoff, (void *)flag, (void *)gnum, (void *)bh,
                        (void *)boff, (void *)bsum, (void *)tags, (void *)err, (void *)bigrows, (void *)nbig})
            cudaFree(q);
        cudaFreeHost(ngroups_h);
        cudaFreeHost(nbig_h);
        if (st) cudaStreamDestroy(st);
    }

    int init(const conan_fof_params &p) {
        R = p.dim;
        device = p.device;
        n = (size_t)p.n_particles;
        // transverse cells no smaller than the linking length (with a margin
        // far above the rounding of the wrap), at most about eight rows per
        // particle
        const double q = p.size / (p.linking_length * (1.0 + 1e-9));
        long long nr = q >= 2147483647.0 ? 2147483647LL : (long long)q;
        long long cap = 1;
        while (true) {
            long long c1 = cap + 1, v = 1;
            for (int k = 1; k < R; ++k) v *= c1;
            if (v > 8 * (long long)std::max<size_t>(n, 27) || v > (1LL << 26)) break;
            cap = c1;
        }
        nr = std::min(nr, cap);
        if (nr < 3) nr = 1;
        g.nr = (int)nr;
        g.L = p.size;
        g.half = p.size / 2;
        g.inv_h = (double)nr / p.size;
        g.xscale = (double)FOF_XN / p.size;
        g.rsqr = p.linking_length * p.linking_length;
        const double wq = std::ceil(p.linking_length * g.xscale) + 2.0;
        g.wq = wq >= (double)FOF_XN ? (int)FOF_XN : (int)wq;
        rows = 1;
        for (int k = 1; k < R; ++k) rows *= (size_t)nr;
        int rb = 0;
        while (((size_t)1 << rb) < rows) ++rb;
        key_bits = FOF_XB + rb;
        const size_t tiles = radix_tiles(n), m = 256 * tiles;
        const size_t nb = (std::max(std::max(m, rows), n) + SCAN_CHUNK - 1) / SCAN_CHUNK;
        CONAN_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        CONAN_CUDA(cudaMalloc(&X, n * R * sizeof(double)));
        CONAN_CUDA(cudaMalloc(&S, n * R * sizeof(double)));
        for (int b = 0; b < 2; ++b) {
            CONAN_CUDA(cudaMalloc(&keys[b], n * sizeof(uint64_t)));
            CONAN_CUDA(cudaMalloc(&vals[b], n * sizeof(uint32_t)));
        }
        CONAN_CUDA(cudaMalloc(&par, n * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&flag, n * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&gnum, (n + 1) * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&rowcount, rows * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&rowoff, (rows + 1) * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&bh, m * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&boff, (m + 1) * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&bsum, nb * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&tags, n * sizeof(unsigned long long)));
        CONAN_CUDA(cudaMalloc(&err, sizeof(int)));
        CONAN_CUDA(cudaMallocHost(&ngroups_h, 2 * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&bigrows, std::min(rows, n / 33 + 1) * sizeof(uint32_t)));
        CONAN_CUDA(cudaMalloc(&nbig, 2 * sizeof(uint32_t)));
        CONAN_CUDA(cudaMallocHost(&nbig_h, 2 * sizeof(uint32_t)));
        int sms = 0;
        CONAN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        sort_blocks = 8 * sms;
        CONAN_CUDA(cudaFuncSetAttribute(k_rs_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS_SMEM));
        CONAN_CUDA(cudaMemsetAsync(rowcount, 0, rows * sizeof(uint32_t), st));
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
        // per-particle keys into keys[1], ranks in the rows into `flag`
        k_fof_keys<RR><<<blocks(n), FOF_T, 0, s>>>(Xd, n, g, keys[1], flag, rowcount);
        scan(rowcount, rows, rowoff, s);  // also clears the counts for the next run
        // counting sort by row, then every row sorted by (x, index)
        CONAN_CUDA(cudaMemsetAsync(nbig, 0, 2 * sizeof(uint32_t), s));
        k_fof_place<<<blocks(n), FOF_T, 0, s>>>(keys[1], flag, rowoff, n, keys[0], vals[0]);
        k_fof_rowsort_small<<<(unsigned)sort_blocks, 256, 0, s>>>(keys[0], vals[0], rowoff, rows, bigrows, nbig);
        k_fof_rowsort_big<<<(unsigned)sort_blocks, 256, 0, s>>>(keys[0], vals[0], rowoff, bigrows, nbig);
        CONAN_CUDA(cudaMemcpyAsync(nbig_h, nbig, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        CONAN_CUDA(cudaStreamSynchronize(s));
        uint64_t *sk = keys[0];
        uint32_t *order = vals[0], *root = vals[1];
        used_radix = nbig_h[1] != 0;
        if (used_radix) {
            // a row longer than FOF_BIG: radix sort of (key, index) from particle order instead
            k_fof_iota<<<blocks(n), FOF_T, 0, s>>>(vals[1], n);
            uint64_t *kk[2] = {keys[1], keys[0]};
            uint32_t *vv[2] = {vals[1], vals[0]};
            const int w = radix_sort_pairs(kk, vv, n, key_bits, bh, boff, bsum, s);
            sk = kk[w];
            order = vv[w];
            root = vv[w ^ 1];
        }
        k_fof_gather<RR><<<blocks(n), FOF_T, 0, s>>>(Xd, n, order, S, par);
        FofLink a{S, sk, order, rowoff, n, g, par, err};
        k_fof_link<RR><<<blocks(n), FOF_T, 0, s>>>(a);
        // roots into the free value buffer, root flags, group numbers
        k_fof_roots<<<blocks(n), FOF_T, 0, s>>>(par, n, root, flag);
        scan(flag, n, gnum, s);
        k_fof_tags<<<blocks(n), FOF_T, 0, s>>>(root, gnum, n, tg);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess)
            return set_error(CONAN_ERR_CUDA, "fof kernel launch failed: %s", cudaGetErrorString(e));
        int herr = 0;
        CONAN_CUDA(cudaMemcpyAsync(ngroups_h, gnum + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
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
