// pm_kernels.cuh -- sm_100a kernels of the particle-mesh step.
//
// Particle state (structure of arrays, one array per axis):
//   d[k][i]  displacement of particle i from its lattice point, in force-mesh
//            cells; the lattice point q = f * (i_0, i_1, i_2) is implicit in i
//            (i_0 fastest), so positions never lose bits to box coordinates.
//   p[k][i]  momentum in force-mesh cells (the reference's P / res_f).
// The reference's absolute position is X = (q + d) * res_f and its momentum
// P = p * res_f (src/run/nbody.hh:46-50,88-95).
//
// Deposit (md_cic, src/run/numeric.hh:106-139) runs as a counting sort by
// cell id followed by a tiled shared-memory reduction:
//   rank   : cell id of every particle (integer, periodic wrap), rank within
//            its cell from an integer counter (fused into the drift),
//   scan   : exclusive prefix of the per-cell counts -> cell offsets,
//   scatter: the particle's cell fractions written at offset + rank,
//   reduce : one CTA per output tile stages the tile's cell offsets in
//            shared memory and walks the sorted particles of its source
//            cells in equal slices; the 2^R corner weights of each particle
//            are quantised to integers, summed per cell in registers and
//            flushed into integer tile accumulators. All sums are integer, so
//            the density is bit-identical from run to run whatever order the
//            sort produced inside a cell; no floating-point atomics are used.
// Every kernel also handles a batch of equal boxes stored back to back
// (ensembles): the member index sits in the high bits of particle and cell
// indices.
#pragma once

#include <climits>

#include "common.cuh"
#include "scan.cuh"

namespace conan {

// Particles of a batch of boxes: particle i belongs to member i >> bshift
// and sits at lattice point i & ((1 << bshift) - 1) of that member.
template <typename T> struct Parts {
    T *d[3];
    T *p[3];
    size_t np;   // whole batch
    int mshift;  // log2(N_m)
    int f;       // force cells per lattice spacing
    int bshift;  // R * mshift
};

// First global force-mesh cell of particle i's member.
template <typename T>
__host__ __device__ inline size_t cell_base(const Parts<T> &P, const Mesh &m, size_t i) {
    return (i >> P.bshift) << m.cshift;
}

template <typename T, int R>
__device__ inline void lattice(const Parts<T> &P, size_t i, int *q) {
    const size_t mmask = ((size_t)1 << P.mshift) - 1;
#pragma unroll
    for (int k = 0; k < R; ++k) q[k] = (int)((i >> (k * P.mshift)) & mmask) * P.f;
}

// ---------------------------------------------------------- payloads --

// FP32: the deposit position is the displacement rounded to 2^-21 cell; the
// three 21-bit cell fractions are packed in one 64-bit word.
// FP64: cell = floor(d), the fractions are kept as doubles.
template <typename T> struct Pay;

template <> struct Pay<float> {
    typedef unsigned long long elem;
    static constexpr int words = 1;
    __device__ static inline void cell_frac(float d, int q, int mask, int *cell, uint32_t *fr) {
        long long Q = __float2ll_rn(d * 2097152.0f);
        *cell = (q + (int)(Q >> 21)) & mask;
        *fr = (uint32_t)(Q & 0x1FFFFF);
    }
};

template <> struct Pay<double> {
    typedef double elem;
    static constexpr int words = 3;
    __device__ static inline void cell_frac(double d, int q, int mask, int *cell, double *fr) {
        double fl = floor(d);
        *cell = (q + (int)fl) & mask;
        *fr = d - fl;
    }
};

// Cell id (axis 0 fastest) of particle i's deposit position.
template <typename T, int R>
__device__ inline uint32_t deposit_cell(const Parts<T> &P, const Mesh &m, size_t i) {
    int q[3];
    lattice<T, R>(P, i, q);
    uint32_t c = 0;
#pragma unroll
    for (int k = R - 1; k >= 0; --k) {
        int ck;
        if constexpr (sizeof(T) == 4) {
            uint32_t fr;
            Pay<float>::cell_frac(P.d[k][i], q[k], m.n - 1, &ck, &fr);
        } else {
            double fr;
            Pay<double>::cell_frac(P.d[k][i], q[k], m.n - 1, &ck, &fr);
        }
        c = (c << m.shift) | (uint32_t)ck;
    }
    return c;
}

// ---------------------------------------------- integer accumulators --

// Corner weights w in [0,1] are rounded to multiples of 2^-23 (FP32) or
// 2^-52 (FP64) with one fused multiply-add onto 2^23 / 2^52 (the rounded
// integer lands in the mantissa), and summed exactly as integers.
struct U128 {
    unsigned long long lo, hi;
};
__device__ inline U128 operator+(U128 a, U128 b) {
    U128 r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
    return r;
}

template <typename T> struct Acc;
template <> struct Acc<float> {
    typedef unsigned long long type;
    __device__ static inline uint32_t quant(float w) {
        return __float_as_uint(__fmaf_rn(w, 8388608.0f, 8388608.0f)) - 0x4B000000u;
    }
    __device__ static inline double value(type s) { return (double)s * 0x1p-23; }
    __device__ static inline type zero() { return 0ull; }
};
template <> struct Acc<double> {
    typedef U128 type;
    __device__ static inline unsigned long long quant(double w) {
        return (unsigned long long)(__double_as_longlong(
                   __fma_rn(w, 4503599627370496.0, 4503599627370496.0)) -
               0x4330000000000000LL);
    }
    __device__ static inline double value(type s) {
        return ((double)s.hi * 0x1p64 + (double)s.lo) * 0x1p-52;
    }
    __device__ static inline type zero() { return U128{0ull, 0ull}; }
};

// ------------------------------------------------------------ rank --

// Counting-sort histogram: cell of every particle and its rank in the cell.
template <typename T, int R>
__global__ void __launch_bounds__(256) k_rank(Parts<T> P, Mesh m, uint32_t *__restrict__ count,
                                              uint32_t *__restrict__ rank) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    uint32_t c = deposit_cell<T, R>(P, m, i);
    rank[i] = atomicAdd(count + cell_base(P, m, i) + c, 1u);
}

// ---------------------------------------------------------- scatter --

// Writes every particle's cell fractions at its sorted slot; optionally the
// particle index too (used by the adjoint's vector deposit).
template <typename T, int R>
__global__ void __launch_bounds__(256) k_scatter(Parts<T> P, Mesh m, const uint32_t *__restrict__ off,
                                                 const uint32_t *__restrict__ rank,
                                                 typename Pay<T>::elem *__restrict__ pay,
                                                 uint32_t *__restrict__ sorted_idx) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    int q[3];
    lattice<T, R>(P, i, q);
    uint32_t c = 0;
    if constexpr (sizeof(T) == 4) {
        unsigned long long word = 0;
#pragma unroll
        for (int k = R - 1; k >= 0; --k) {
            int ck;
            uint32_t fr;
            Pay<float>::cell_frac(P.d[k][i], q[k], m.n - 1, &ck, &fr);
            c = (c << m.shift) | (uint32_t)ck;
            word |= (unsigned long long)fr << (21 * k);
        }
        uint32_t dst = off[cell_base(P, m, i) + c] + rank[i];
        if (dst >= P.np) return;  // unreachable when counts and ranks agree
        pay[dst] = word;
        if (sorted_idx) sorted_idx[dst] = (uint32_t)i;
    } else {
        double fr[3];
#pragma unroll
        for (int k = R - 1; k >= 0; --k) {
            int ck;
            Pay<double>::cell_frac(P.d[k][i], q[k], m.n - 1, &ck, &fr[k]);
            c = (c << m.shift) | (uint32_t)ck;
        }
        uint32_t dst = off[cell_base(P, m, i) + c] + rank[i];
        if (dst >= P.np) return;  // unreachable when counts and ranks agree
#pragma unroll
        for (int k = 0; k < R; ++k) pay[(size_t)dst * R + k] = fr[k];
        if (sorted_idx) sorted_idx[dst] = (uint32_t)i;
    }
}

// Cell fractions of sorted particle j.
template <typename T, int R>
__device__ inline void load_frac(const typename Pay<T>::elem *__restrict__ pay, uint32_t j, T *fr) {
    if constexpr (sizeof(T) == 4) {
        unsigned long long w = pay[j];
#pragma unroll
        for (int k = 0; k < R; ++k) fr[k] = (float)((uint32_t)(w >> (21 * k)) & 0x1FFFFFu) * 0x1p-21f;
    } else {
#pragma unroll
        for (int k = 0; k < R; ++k) fr[k] = pay[(size_t)j * R + k];
    }
}

// CIC weight of corner b (bit k of b = +1 along axis k) from the fractions.
template <typename T, int R> __device__ inline T corner_weight(const T *fr, int b) {
    T z = 1;
#pragma unroll
    for (int k = 0; k < R; ++k) z *= ((b >> k) & 1) ? fr[k] : (T(1) - fr[k]);
    return z;
}

// ------------------------------------------------------ deposit reduce --

// Tile accumulators of the deposit: W 32-bit words per cell stored as W
// planes of CELLS words (so lanes flushing neighbouring cells hit distinct
// banks), updated with native 32-bit shared atomics and explicit carries.
// FP32: 64-bit sums in units of 2^-23. FP64: 96-bit sums in units of 2^-52.
template <typename T> struct Slot;
template <> struct Slot<float> {
    static constexpr int W = 2;
    __device__ static inline void add(uint32_t *s, int c, uint32_t v, int cells) {
        if (!v) return;
        uint32_t old = atomicAdd(s + c, v);
        if (old + v < old) atomicAdd(s + cells + c, 1u);
    }
    __device__ static inline double value(const uint32_t *s, int c, int cells) {
        return ((double)s[cells + c] * 4294967296.0 + (double)s[c]) * 0x1p-23;
    }
};
template <> struct Slot<double> {
    static constexpr int W = 3;
    __device__ static inline void add(uint32_t *s, int c, unsigned long long v, int cells) {
        if (!v) return;
        uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);  // hi < 2^31
        uint32_t old = atomicAdd(s + c, lo);
        uint32_t x = hi + (old + lo < old ? 1u : 0u);
        if (!x) return;
        uint32_t old1 = atomicAdd(s + cells + c, x);
        if (old1 + x < old1) atomicAdd(s + 2 * cells + c, 1u);
    }
    __device__ static inline double value(const uint32_t *s, int c, int cells) {
        return (double)s[2 * cells + c] * 0x1p12 + (double)s[cells + c] * 0x1p-20 + (double)s[c] * 0x1p-52;
    }
};

// Per-thread register sums of the 2^R corner weights of one source cell.
template <typename T> struct RegAcc;
template <> struct RegAcc<float> {
    typedef uint32_t type;                 // <= 2^23 per particle
    static constexpr int max_terms = 511;  // 511 * 2^23 < 2^32
};
template <> struct RegAcc<double> {
    typedef unsigned long long type;        // <= 2^52 per particle
    static constexpr int max_terms = 2047;  // 2047 * 2^52 < 2^63
};

__device__ inline uint32_t quant_w(float w) {
    return __float_as_uint(__fmaf_rn(w, 8388608.0f, 8388608.0f)) - 0x4B000000u;
}
__device__ inline unsigned long long quant_w(double w) {
    return (unsigned long long)(__double_as_longlong(__fma_rn(w, 4503599627370496.0, 4503599627370496.0)) -
                                0x4330000000000000LL);
}

// Tile shape of the deposit for dimension R: TX x TY x TZ output cells.
// Variant V (0 = default) of the tile shape; the autotuner picks one per
// mesh size.
constexpr int DEP_VARIANTS = 3;
template <int R, int V = 0> struct DepTile;
template <> struct DepTile<3, 0> { static constexpr int TX = 32, TY = 8, TZ = 8, THREADS = 256; };
template <> struct DepTile<3, 1> { static constexpr int TX = 32, TY = 4, TZ = 8, THREADS = 128; };
template <> struct DepTile<3, 2> { static constexpr int TX = 32, TY = 16, TZ = 8, THREADS = 512; };
template <> struct DepTile<2, 0> { static constexpr int TX = 32, TY = 32, TZ = 1, THREADS = 256; };
template <> struct DepTile<2, 1> { static constexpr int TX = 32, TY = 16, TZ = 1, THREADS = 128; };
template <> struct DepTile<2, 2> { static constexpr int TX = 64, TY = 32, TZ = 1, THREADS = 512; };
template <> struct DepTile<1, 0> { static constexpr int TX = 1024, TY = 1, TZ = 1, THREADS = 256; };
template <> struct DepTile<1, 1> { static constexpr int TX = 512, TY = 1, TZ = 1, THREADS = 128; };
template <> struct DepTile<1, 2> { static constexpr int TX = 2048, TY = 1, TZ = 1, THREADS = 512; };

// One CTA deposits one output tile. Its source cells are the tile plus one
// cell on the low side of every axis (a particle in cell s reaches s..s+1).
// The sorted particles of those source cells form (TY+1)(TZ+1) contiguous
// row ranges; the CTA stages their cell offsets in shared memory, splits the
// concatenated particle list into equal contiguous slices (one per thread,
// load-balanced whatever the clustering), and each thread sums the corner
// weights of consecutive particles of one cell in registers, flushing to the
// tile's integer accumulators when the cell changes. Integer sums make the
// result independent of the order of particles and flushes.
template <typename T, int R, int TX, int TY, int TZ, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
    k_deposit(const uint32_t *__restrict__ off, const typename Pay<T>::elem *__restrict__ pay,
              T *__restrict__ out, Mesh m, double scale, uint32_t np, int *__restrict__ err) {
    constexpr int HY = R >= 2 ? 1 : 0, HZ = R == 3 ? 1 : 0;
    constexpr int NR = (TY + HY) * (TZ + HZ);  // source rows
    constexpr int RAW = TX + 3;                 // hb, he, off[x0 .. x0+TX]
    constexpr int CELLS = TX * TY * TZ;
    constexpr int C = 1 << R;
    extern __shared__ __align__(16) unsigned char dep_sh[];
    uint32_t *slot = reinterpret_cast<uint32_t *>(dep_sh);
    uint32_t *raw = slot + Slot<T>::W * CELLS;
    uint32_t *rp = raw + NR * RAW;  // NR + 1 row prefixes

    const int n = m.n, mask = n - 1;
    const int ntx = n / TX, nty = R >= 2 ? n / TY : 1, ntz = R == 3 ? n / TZ : 1;
    const int tiles = ntx * nty * ntz;  // per member of the batch
    const size_t mbase = member_cells(m, blockIdx.x / tiles);
    off += mbase;
    out += mbase;
    const int tile = blockIdx.x % tiles;
    const int x0 = (tile % ntx) * TX;
    const int y0 = R >= 2 ? ((tile / ntx) % nty) * TY : 0;
    const int z0 = R == 3 ? (tile / (ntx * nty)) * TZ : 0;
    const int hx = (x0 - 1) & mask;

    for (int c = threadIdx.x; c < Slot<T>::W * CELLS; c += THREADS) slot[c] = 0u;
    for (int i = threadIdx.x; i < NR * RAW; i += THREADS) {
        int r = i / RAW, k = i % RAW;
        int ry = r % (TY + HY), rz = r / (TY + HY);
        int y = (y0 - HY + ry) & mask, z = (z0 - HZ + rz) & mask;
        size_t rb = 0;
        if (R == 2) rb = (size_t)y << m.shift;
        if (R == 3) rb = ((size_t)z << (2 * m.shift)) | ((size_t)y << m.shift);
        size_t idx = k == 0 ? rb + hx : k == 1 ? rb + hx + 1 : rb + x0 + (k - 2);
        raw[i] = __ldg(off + idx);
    }
    __syncthreads();

    // Row totals (validated) and their exclusive prefix, by warp 0.
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t run = 0;
        for (int base = 0; base < NR; base += 32) {
            int r = base + lane;
            uint32_t tot = 0;
            if (r < NR) {
                const uint32_t *w = raw + r * RAW;
                bool ok = w[1] >= w[0] && w[TX + 2] >= w[2];
                tot = ok ? (w[1] - w[0]) + (w[TX + 2] - w[2]) : 0u;
                if (!ok) atomicOr(err, 2);
            }
            uint32_t inc = tot;
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t v = __shfl_up_sync(FULL, inc, o);
                if (lane >= o) inc += v;
            }
            if (r < NR) rp[r] = run + inc - tot;
            run += __shfl_sync(FULL, inc, 31);
        }
        // halo rows/columns repeat cells when a tile spans the whole mesh,
        // so a valid total is at most 2^R times the particle count
        bool bad = (unsigned long long)run > ((unsigned long long)np << R);
        if (lane == 0) rp[NR] = bad ? 0u : run;
        if (lane == 0 && bad) atomicOr(err, 2);
    }
    __syncthreads();

    const uint32_t total = rp[NR];
    const uint32_t P = (total + THREADS - 1) / THREADS;
    uint32_t g = threadIdx.x * P;
    const uint32_t gend = min(g + P, total);
    if (g < gend) {
        // starting row: last r with rp[r] <= g
        int r = 0;
        for (int step = 512; step >= 1; step >>= 1)
            if (r + step <= NR - 1 && rp[r + step] <= g) r += step;
        while (r < NR - 1 && rp[r + 1] <= g) ++r;
        const uint32_t *w = raw + r * RAW;
        uint32_t hb = w[0], hc = w[1] - w[0], b0 = w[2];
        uint32_t j = g - rp[r];
        uint32_t rowtot = rp[r + 1] - rp[r];
        // logical cell m: 0 = halo x0-1, 1 + L = cell x0 + L;
        // boundary B(m) = 0 (m = 0), hc + w[m + 1] - b0 (m >= 1)
        int mc = 0;
        while (mc < TX && hc + (w[mc + 2] - b0) <= j) ++mc;
        uint32_t nb = hc + (w[mc + 2] - b0);  // end of cell mc
        typename RegAcc<T>::type acc[C];
#pragma unroll
        for (int b = 0; b < C; ++b) acc[b] = 0;
        int terms = 0;

#define CONAN_DEP_FLUSH()                                                                   \
    do {                                                                                    \
        if (terms) {                                                                        \
            int ry_ = r % (TY + HY), rz_ = r / (TY + HY);                                  \
            int sx_ = mc - 1, sy_ = ry_ - HY, sz_ = rz_ - HZ;                              \
            _Pragma("unroll") for (int b = 0; b < C; ++b) {                                 \
                int ox = sx_ + (b & 1);                                                     \
                int oy = R >= 2 ? sy_ + ((b >> 1) & 1) : 0;                                 \
                int oz = R == 3 ? sz_ + ((b >> 2) & 1) : 0;                                 \
                if (ox >= 0 && ox < TX && oy >= 0 && oy < TY && oz >= 0 && oz < TZ)         \
                    Slot<T>::add(slot, (oz * TY + oy) * TX + ox, acc[b], CELLS);             \
                acc[b] = 0;                                                                 \
            }                                                                               \
            terms = 0;                                                                      \
        }                                                                                   \
    } while (0)

        for (; g < gend; ++g, ++j) {
            while (j >= rowtot) {  // next non-empty row
                CONAN_DEP_FLUSH();
                ++r;
                w = raw + r * RAW;
                hb = w[0];
                hc = w[1] - w[0];
                b0 = w[2];
                j = 0;
                rowtot = rp[r + 1] - rp[r];
                mc = 0;
                nb = hc;
            }
            while (j >= nb && mc < TX) {  // next non-empty cell of the row
                CONAN_DEP_FLUSH();
                ++mc;
                nb = hc + (w[mc + 2] - b0);
            }
            if (j >= nb) {  // non-monotone offsets: unreachable, never walk on
                atomicOr(err, 4);
                break;
            }
            uint32_t src = mc == 0 ? hb + j : b0 + (j - hc);
            if (src >= np) {  // unreachable with valid offsets
                atomicOr(err, 1);
                continue;
            }
            T fr[3];
            load_frac<T, R>(pay, src, fr);
            T g0 = T(1) - fr[0];
            T wx[2] = {g0, fr[0]};
            T wy[2] = {T(1), T(1)}, wz[2] = {T(1), T(1)};
            if (R >= 2) {
                wy[0] = T(1) - fr[1];
                wy[1] = fr[1];
            }
            if (R == 3) {
                wz[0] = T(1) - fr[2];
                wz[1] = fr[2];
            }
#pragma unroll
            for (int b = 0; b < C; ++b) {
                T wb = wx[b & 1] * wy[(b >> 1) & 1] * wz[(b >> 2) & 1];
                acc[b] += quant_w(wb);
            }
            if (++terms == RegAcc<T>::max_terms) CONAN_DEP_FLUSH();
        }
        CONAN_DEP_FLUSH();
    }
#undef CONAN_DEP_FLUSH
    __syncthreads();

    for (int c = threadIdx.x; c < CELLS; c += THREADS) {
        int ox = c % TX, oy = (c / TX) % TY, oz = c / (TX * TY);
        size_t o = (size_t)(x0 + ox);
        if (R >= 2) o |= (size_t)(y0 + oy) << m.shift;
        if (R == 3) o |= (size_t)(z0 + oz) << (2 * m.shift);
        out[o] = (T)(Slot<T>::value(slot, c, CELLS) * scale - 1.0);
    }
}

template <typename T, int R, int V = 0> constexpr size_t deposit_smem() {
    typedef DepTile<R, V> D;
    constexpr int HY = R >= 2 ? 1 : 0, HZ = R == 3 ? 1 : 0;
    constexpr int NR = (D::TY + HY) * (D::TZ + HZ);
    return sizeof(uint32_t) * (Slot<T>::W * D::TX * D::TY * D::TZ + NR * (D::TX + 3) + NR + 1);
}

__device__ inline void acc_add(unsigned long long &a, unsigned long long v) { a += v; }
__device__ inline void acc_add(U128 &a, unsigned long long v) { a = a + U128{v, 0ull}; }

// Reference kernel for small meshes (n < 32): one thread per output cell
// pulls the particles of its 2^R source cells. Same integer sums.
template <typename T, int R>
__global__ void k_deposit_pull(const uint32_t *__restrict__ off,
                               const typename Pay<T>::elem *__restrict__ pay, T *__restrict__ out,
                               Mesh m, double scale) {
    size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.cells) return;
    int x[3] = {0, 0, 0};
    for (int k = 0; k < R; ++k) x[k] = (int)((c >> (k * m.shift)) & (size_t)(m.n - 1));
    typename Acc<T>::type s = Acc<T>::zero();
    for (int b = 0; b < (1 << R); ++b) {
        size_t sc = 0;
        for (int k = R - 1; k >= 0; --k)
            sc = (sc << m.shift) | (size_t)((x[k] - ((b >> k) & 1)) & (m.n - 1));
        sc += member_cells(m, c >> m.cshift);
        for (uint32_t j = off[sc]; j < off[sc + 1]; ++j) {
            T fr[3];
            load_frac<T, R>(pay, j, fr);
            acc_add(s, Acc<T>::quant(corner_weight<T, R>(fr, b)));
        }
    }
    out[c] = (T)(Acc<T>::value(s) * scale - 1.0);
}

// ------------------------------------------------------------ Poisson --

// Green's function multiply on the half spectrum: spec *= gs / |n|^2 with
// gs = -G/(a N_c) (L/2pi)^2, DC = 0 (src/run/nbody.hh:105-110 with
// Fourier::potential, src/base/fourier.hh:102-109).
// One CTA per row of the half spectrum (n/2 + 1 elements along kx): the
// row's ky, kz come from the block index by bit operations, so no element
// index is ever divided.
template <typename T>
__global__ void __launch_bounds__(256) k_green(typename Cplx<T>::type *__restrict__ spec, Mesh m, T gs) {
    const size_t row = blockIdx.x;  // n^(R-1) rows per member, members back to back
    long long kyz = 0;
    for (int a = 1; a < m.R; ++a) {
        const int ia = (int)((row >> ((a - 1) * m.shift)) & (size_t)(m.n - 1));
        const int w = wave_index(ia, m.n);
        kyz += (long long)w * w;
    }
    typename Cplx<T>::type *r = spec + row * (size_t)m.nh;
    for (int kx = threadIdx.x; kx < m.nh; kx += blockDim.x) {
        const long long k2 = (long long)kx * kx + kyz;
        T g = k2 > 0 ? gs / (T)k2 : T(0);
        auto z = r[kx];
        z.x *= g;
        z.y *= g;
        r[kx] = z;
    }
}

// Spectral derivative along `axis` in cell units: out = i (2 pi n_axis / n)
// in, zero on the axis' Nyquist plane.
template <typename T>
__global__ void k_spec_deriv(const typename Cplx<T>::type *__restrict__ in,
                             typename Cplx<T>::type *__restrict__ out, Mesh m, int axis) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.spec) return;
    int kv[3];
    spec_k2(e, m, kv);
    int ka = kv[axis];
    T s = (2 * ka == m.n || 2 * ka == -m.n) ? T(0) : (T)(2.0 * M_PI / m.n) * (T)ka;
    auto z = in[e];
    typename Cplx<T>::type r;
    r.x = -z.y * s;
    r.y = z.x * s;
    out[e] = r;
}

// --------------------------------------------------- gather/kick/drift --

// 4-point central difference of f along axis k at cell c, in units of
// f per cell (Gradient<R>::operator[], src/run/numeric.hh:88-100).
template <typename T, int R>
__device__ inline T fd4(const T *__restrict__ f, const int *c, int k, int shift, int mask) {
    size_t base = 0;
#pragma unroll
    for (int a = R - 1; a >= 0; --a)
        if (a != k) base |= (size_t)c[a] << (a * shift);
    auto at = [&](int o) { return __ldg(f + (base | ((size_t)((c[k] + o) & mask) << (k * shift)))); };
    const T c12 = T(1) / T(12), c23 = T(2) / T(3);
    return (at(-2) - at(2)) * c12 + (at(1) - at(-1)) * c23;
}

// Gather origin and weights along one axis: the reference interpolates at
// x = X / res with origin = (int)x (truncation toward zero), so particles
// at negative unwrapped coordinates get extrapolated weights
// (src/run/numeric.hh:19-29). periodic = true uses floor instead.
template <typename T>
__device__ inline void gather_axis(T d, int q, bool periodic, int *o, T *a1) {
    T fl = floor(d);
    int org = q + (int)fl;
    T fr = d - fl;
    if (!periodic && org < 0 && fr != T(0)) {
        org += 1;
        fr -= T(1);
    }
    *o = org;
    *a1 = fr;
}

// Packed gradient of one mesh node (x, y, z, unused).
template <typename T> struct alignas(16) G4 {
    T x, y, z, w;
};
__device__ inline G4<float> load_g4(const G4<float> *p) {
    float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    return G4<float>{v.x, v.y, v.z, v.w};
}
__device__ inline G4<double> load_g4(const G4<double> *p) {
    double2 a = __ldg(reinterpret_cast<const double2 *>(p));
    double2 b = __ldg(reinterpret_cast<const double2 *>(p) + 1);
    return G4<double>{a.x, a.y, b.x, b.y};
}

// The FD4 gradient of phi at every node, in units of phi per cell, packed:
// the reference's Gradient<R>::operator[] (src/run/numeric.hh:88-100)
// evaluated once per node for all particles that interpolate it.
template <typename T, int R>
__global__ void __launch_bounds__(512) k_fd_grad(const T *__restrict__ phi, G4<T> *__restrict__ G, Mesh m) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.cells) return;
    const uint32_t mask = m.n - 1;
    const T c12 = T(1) / T(12), c23 = T(2) / T(3);
    T g[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const int sh = k * m.shift;
        uint32_t ck = (c >> sh) & mask, rest = c & ~(mask << sh);
        auto at = [&](int o) { return __ldg(phi + (rest | (((ck + o) & mask) << sh))); };
        g[k] = (at(-2) - at(2)) * c12 + (at(1) - at(-1)) * c23;
    }
    G[c] = G4<T>{g[0], g[1], g[2], T(0)};
}

// The same gradient for 3D meshes of at least 32 cells per side, marching
// along z: a CTA of 32 x 8 threads takes a 32 x 8 column of cells over FZ
// planes. Each plane's tile with a two-cell halo in x and y is staged in
// shared memory (two buffers, one barrier per plane, the next plane's loads
// in flight while a plane is computed) for the x and y differences, and
// each thread keeps its column's five z values in registers; the same
// arithmetic as k_fd_grad, so the same bits.
#ifndef FD_GRAD_ZM
#define FD_GRAD_ZM 0
#endif
constexpr int FDZ_PLANES = 16;

template <typename T>
__global__ void __launch_bounds__(256) k_fd_grad_zm(const T *__restrict__ phi, G4<T> *__restrict__ G, Mesh m) {
    __shared__ T tile[2][12][36];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const uint32_t mask = (uint32_t)m.n - 1;
    const int s = m.shift;
    const int nbx = m.n >> 5, nby = m.n >> 3, nbz = m.n / FDZ_PLANES;
    unsigned b = blockIdx.x;
    const int bx = (int)(b % nbx);
    b /= nbx;
    const int by = (int)(b % nby);
    b /= nby;
    const int bz = (int)(b % nbz);
    const size_t mb = (size_t)(b / nbz) << m.cshift;
    const T *__restrict__ ph = phi + mb;
    G4<T> *__restrict__ g = G + mb;
    const int x0 = bx * 32, y0 = by * 8, z0 = bz * FDZ_PLANES;
    auto at = [&](int xx, int yy, int zz) {
        return __ldg(ph + (((size_t)((uint32_t)zz & mask) << (2 * s)) | (((uint32_t)yy & mask) << s) |
                           ((uint32_t)xx & mask)));
    };
    const T c12 = T(1) / T(12), c23 = T(2) / T(3);
    T q[5];  // this column at z - 2 .. z + 2
#pragma unroll
    for (int j = 0; j < 5; ++j) q[j] = at(x0 + tx, y0 + ty, z0 - 2 + j);
    // this thread's share of a plane's 12 x 36 halo tile (elements threadIdx,
    // threadIdx + 256): the next plane's share is loaded while this plane is
    // computed, and stored into the other buffer at the top of the next
    // iteration (the barrier of this iteration orders it after every read of
    // that buffer two planes back)
    constexpr int TE = 12 * 36;
    auto tile_at = [&](int e, int zz) {
        const int r = e / 36, c = e - r * 36;
        return at(x0 - 2 + c, y0 - 2 + r, zz);
    };
    T nxt[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int e = (int)threadIdx.x + 256 * k;
        nxt[k] = e < TE ? tile_at(e, z0) : T(0);
    }
    for (int zi = 0; zi < FDZ_PLANES; ++zi) {
        const int z = z0 + zi;
        T(*t)[36] = tile[zi & 1];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const int e = (int)threadIdx.x + 256 * k;
            if (e < TE) t[e / 36][e % 36] = nxt[k];
        }
        __syncthreads();
        T q4n = T(0);
        if (zi + 1 < FDZ_PLANES) {
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int e = (int)threadIdx.x + 256 * k;
                if (e < TE) nxt[k] = tile_at(e, z + 1);
            }
            q4n = at(x0 + tx, y0 + ty, z + 3);
        }
        const T gx = (t[ty + 2][tx] - t[ty + 2][tx + 4]) * c12 + (t[ty + 2][tx + 3] - t[ty + 2][tx + 1]) * c23;
        const T gy = (t[ty][tx + 2] - t[ty + 4][tx + 2]) * c12 + (t[ty + 3][tx + 2] - t[ty + 1][tx + 2]) * c23;
        const T gz = (q[0] - q[4]) * c12 + (q[3] - q[1]) * c23;
        g[((size_t)z << (2 * s)) | ((size_t)(y0 + ty) << s) | (size_t)(x0 + tx)] = G4<T>{gx, gy, gz, T(0)};
#pragma unroll
        for (int j = 0; j < 4; ++j) q[j] = q[j + 1];
        q[4] = q4n;
    }
}

// CIC-interpolated force of particle i: sum over corners of weight times
// the node gradient (packed FD4 mesh G, or the spectral gradient meshes g[k]).
template <typename T, int R, bool SPECTRAL>
__device__ inline void gather_force(const Parts<T> &P, const Mesh &m, size_t i, const T *phi,
                                    const T *const *g, const G4<T> *__restrict__ G, bool periodic,
                                    const T *d, T *F) {
    int q[3], o[3];
    T a1[3], a0[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        gather_axis<T>(d[k], q[k], periodic, &o[k], &a1[k]);
        a0[k] = T(1) - a1[k];
        F[k] = T(0);
    }
    const int mask = m.n - 1;
    const size_t cb = cell_base(P, m, i);
    if constexpr (SPECTRAL) {
#pragma unroll
        for (int b = 0; b < (1 << R); ++b) {
            T z = 1;
            size_t ci = 0;
#pragma unroll
            for (int k = R - 1; k >= 0; --k) ci = (ci << m.shift) | (size_t)((o[k] + ((b >> k) & 1)) & mask);
#pragma unroll
            for (int k = 0; k < R; ++k) z *= ((b >> k) & 1) ? a1[k] : a0[k];
#pragma unroll
            for (int k = 0; k < R; ++k) F[k] += __ldg(g[k] + cb + ci) * z;
        }
    } else {
        // FD4 gradient of the corner nodes from the packed gradient mesh
        // (one 16-byte load per corner for FP32).
        (void)phi;
#pragma unroll
        for (int b = 0; b < (1 << R); ++b) {
            uint32_t ci = 0;
#pragma unroll
            for (int k = R - 1; k >= 0; --k) ci = (ci << m.shift) | (uint32_t)((o[k] + ((b >> k) & 1)) & mask);
            T z = 1;
#pragma unroll
            for (int k = 0; k < R; ++k) z *= ((b >> k) & 1) ? a1[k] : a0[k];
            G4<T> gv = load_g4(G + cb + ci);
            F[0] += gv.x * z;
            if (R > 1) F[1] += gv.y * z;
            if (R > 2) F[2] += gv.z * z;
        }
    }
}

// Particle index of thread `tid` of block `blk` when the lattice is walked in
// compact tiles (16x4x4 in 3D, 32x8 in 2D) so that a block's particles,
// and so their potential reads, stay close together; linear otherwise.
template <typename T, int R>
__device__ inline size_t tiled_index(const Parts<T> &P, unsigned blk, unsigned tid) {
    const int s = P.mshift;
    if (R == 3 && s >= 4) {
        size_t tx = blk & ((1u << (s - 4)) - 1), rest = blk >> (s - 4);
        size_t ty = rest & ((1u << (s - 2)) - 1), tz = rest >> (s - 2);
        size_t x = tx * 16 + (tid & 15), y = ty * 4 + ((tid >> 4) & 3), z = tz * 4 + (tid >> 6);
        return x | (y << s) | (z << (2 * s));
    }
    if (R == 2 && s >= 5) {
        size_t tx = blk & ((1u << (s - 5)) - 1), ty = blk >> (s - 5);
        size_t x = tx * 32 + (tid & 31), y = ty * 8 + (tid >> 5);
        return x | (y << s);
    }
    return (size_t)blk * 256 + tid;
}

struct GKD {
    double ck;  // kick: p -= F ck (0 disables)
    double cd;  // drift: d += p cd (after the kick)
    int kick, drift, rank, periodic;
    int deposit = 1;  // fused Lagrangian tiles: deposit the drifted positions (0: kick and/or drift only)
};

// Fused leapfrog update of particle i: the kick of Gravity::kick
// (src/run/nbody.hh:112-117), then the next step's drift (Gravity::drift,
// src/run/nbody.hh:122-130), then the counting-sort rank of the new cell.
template <typename T, int R, bool SPECTRAL>
__global__ void __launch_bounds__(256)
    k_gkd(Parts<T> P, Mesh m, const T *__restrict__ phi, const T *__restrict__ g0,
          const T *__restrict__ g1, const T *__restrict__ g2, const G4<T> *__restrict__ G, GKD c,
          uint32_t *__restrict__ count, uint32_t *__restrict__ rank) {
    size_t i = tiled_index<T, R>(P, blockIdx.x, threadIdx.x);
    if (i >= P.np) return;
    T d[3], p[3];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        d[k] = P.d[k][i];
        p[k] = P.p[k][i];
    }
    if (c.kick) {
        T F[3];
        const T *g[3] = {g0, g1, g2};
        gather_force<T, R, SPECTRAL>(P, m, i, phi, g, G, c.periodic, d, F);
        const T ck = (T)c.ck;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            p[k] -= F[k] * ck;
            P.p[k][i] = p[k];
        }
    }
    if (c.drift) {
        const T cd = (T)c.cd;
#pragma unroll
        for (int k = 0; k < R; ++k) {
            d[k] += p[k] * cd;
            P.d[k][i] = d[k];
        }
    }
    if (c.rank) rank[i] = atomicAdd(count + cell_base(P, m, i) + deposit_cell<T, R>(P, m, i), 1u);
}

// ------------------------------------------------ Lagrangian deposit --
//
// FP32 deposit without the sort. One CTA takes a tile of the particle
// lattice (particles are stored in lattice order, so its loads are
// coalesced), finds the bounding box of the tile's current cells, and sums
// the quantised corner weights of every particle into a shared-memory window
// of the force mesh placed over that box (64-bit integer slots). The window is
// then added into a 64-bit integer accumulator mesh, one add per non-empty
// cell; a particle whose corners leave the window (a tile stretched wider
// than the window) adds its corners to the accumulator directly. Every sum is
// an integer sum, so the density does not depend on the order of the adds
// and equals the sorted deposit bit for bit (same fractions, same quantised
// weights, same final scaling). k_acc_mesh turns the accumulator into the
// density contrast; a memset clears it for the next deposit.

// Window of the Lagrangian deposit: w[k] force cells along axis k (1 beyond
// R); cells = w0 w1 w2 rounded up to a multiple of 4.
struct LagWin {
    int w[3];
    int cells;
};

// Lattice tile (LX x LY x LZ particles), threads and window margin M (cells
// beyond the tile's own f*L cells, split over both sides) of variant V.
constexpr int LAG_VARIANTS = 3;
// 32-bit planes of a window cell: 2 keeps the carry in shared memory, 1
// sends it to the accumulator mesh (a carry needs over 2^9 particles' weight
// in one cell of one tile: rare). A compile-time tunable; one plane leaves
// room for the TMA-staged tile's arrays beside its window (3.55 against 3.76
// ms per fused launch at 512^3).
#ifndef LAG_PLANES
#define LAG_PLANES 1
#endif

// Window cells per particle of a tile above which the deposit goes to the
// accumulator mesh directly (fine meshes); a compile-time tunable.
#ifndef LAG_WINDOW_CELLS_PER_PARTICLE
#define LAG_WINDOW_CELLS_PER_PARTICLE 12.0
#endif

template <int R, int V> struct LagTile;
template <> struct LagTile<3, 0> { static constexpr int LX = 32, LY = 8, LZ = 8, THREADS = 512, M = 8; };
template <> struct LagTile<3, 1> { static constexpr int LX = 16, LY = 8, LZ = 8, THREADS = 256, M = 8; };
template <> struct LagTile<3, 2> { static constexpr int LX = 8, LY = 8, LZ = 8, THREADS = 128, M = 8; };
template <> struct LagTile<2, 0> { static constexpr int LX = 64, LY = 32, LZ = 1, THREADS = 512, M = 16; };
template <> struct LagTile<2, 1> { static constexpr int LX = 32, LY = 16, LZ = 1, THREADS = 128, M = 16; };
template <> struct LagTile<2, 2> { static constexpr int LX = 16, LY = 16, LZ = 1, THREADS = 64, M = 16; };
template <> struct LagTile<1, 0> { static constexpr int LX = 2048, LY = 1, LZ = 1, THREADS = 512, M = 64; };
template <> struct LagTile<1, 1> { static constexpr int LX = 512, LY = 1, LZ = 1, THREADS = 128, M = 64; };
template <> struct LagTile<1, 2> { static constexpr int LX = 128, LY = 1, LZ = 1, THREADS = 32, M = 32; };

// The body of the Lagrangian deposit for one lattice tile. FUSED: the
// particles are first advanced as in k_gkd (gather of the packed gradient,
// kick, drift; positions and momenta written back) and the new positions are
// deposited, so the deposit costs no second pass over the particles.
// STAGED: the tile's d[0..2], p[0..2] arrive in shared memory (six
// LX*LY*LZ arrays in tile order, see k_gkd_lag_tma), particle group j
// signalled by bars[j]; otherwise they are read from global memory.
__device__ inline bool tma_wait(unsigned long long *bar, unsigned limit, unsigned parity = 0);
constexpr unsigned TMA_WAIT_LIMIT = 1u << 20;  // polls of try_wait (about a second at most)

// Deposit position of a displacement d (force cells) along one axis: d
// rounded to 2^-21 cell, Q = rn(d 2^21), cell offset Q >> 21 (floor) and
// fraction Q & (2^21 - 1), as Pay<float>::cell_frac. 32-bit integer
// arithmetic while |d 2^21| < 2^31 (displacements below 1024 cells), 64-bit
// beyond; both give the same integers.
__device__ __forceinline__ void quant_pos(float d, int *cell, uint32_t *fr) {
    const float s = d * 2097152.0f;
    if (fabsf(s) < 2147483648.0f) {
        const int Q = __float2int_rn(s);
        *cell = Q >> 21;
        *fr = (uint32_t)Q & 0x1FFFFFu;
    } else {
        const long long Q = __float2ll_rn(s);
        *cell = (int)(Q >> 21);
        *fr = (uint32_t)(Q & 0x1FFFFF);
    }
}

// CIC force of one particle from the packed FD4 gradient mesh Gm of its
// member (gather_force<float, R, false> with 32-bit corner offsets; same
// operations in the same order): q lattice point in force cells, d its
// displacement.
template <int R>
__device__ __forceinline__ void gather_g4(const G4<float> *__restrict__ Gm, int shift, uint32_t mask, const int *q,
                                          const float *d, bool periodic, float *F) {
    int o[3] = {0, 0, 0};
    float a1[3] = {0.f, 0.f, 0.f}, a0[3] = {1.f, 1.f, 1.f};
#pragma unroll
    for (int k = 0; k < R; ++k) {
        gather_axis<float>(d[k], q[k], periodic, &o[k], &a1[k]);
        a0[k] = 1.0f - a1[k];
    }
    uint32_t off[3][2];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        off[k][0] = k < R ? ((uint32_t)o[k] & mask) << (k * shift) : 0u;
        off[k][1] = k < R ? ((uint32_t)(o[k] + 1) & mask) << (k * shift) : 0u;
    }
    // z = ((1 a_x) a_y) a_z, as the loop of gather_force multiplies
    float wxy[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) wxy[b] = (b & 1 ? a1[0] : a0[0]) * (R >= 2 ? (b & 2 ? a1[1] : a0[1]) : 1.0f);
    F[0] = F[1] = F[2] = 0.0f;
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        const uint32_t ci = off[0][b & 1] + off[1][(b >> 1) & 1] + off[2][(b >> 2) & 1];
        const float z = R == 3 ? wxy[b & 3] * ((b & 4) ? a1[2] : a0[2]) : wxy[b & 3];
        const G4<float> gv = load_g4(Gm + ci);
        F[0] += gv.x * z;
        if (R > 1) F[1] += gv.y * z;
        if (R > 2) F[2] += gv.z * z;
    }
}

// Staged tiles keep the drifted displacements in the staging memory and
// place the window after it (instead of over it): the deposit reads the
// particles back from shared memory, not from registers, and the window is
// cleared while the copies arrive. A compile-time tunable.
#ifndef LAG_STAGE_KEEP
#define LAG_STAGE_KEEP 1
#endif
// The staged fused launches run as persistent CTAs that prefetch their next
// tile (k_gkd_lag_pers) by default; a compile-time tunable, and a knob of
// the autotuner.
#ifndef LAG_PERSIST
#define LAG_PERSIST 0
#endif
// The gather + kick + drift + deposit launches staged too (not only the
// first drift + deposit); a compile-time tunable.
#ifndef LAG_TMA_GATHER
#define LAG_TMA_GATHER 1
#endif

// PERSIST: one tile of a persistent CTA (k_gkd_lag_pers): the tile index,
// the phase parity of this use of the staging buffer's barriers and the
// window (kept clear between tiles: the flush zeroes what it reads) come
// from the caller.
template <int R, int LX, int LY, int LZ, int THREADS, bool FUSED, bool STAGED = false, bool PERSIST = false>
__device__ __forceinline__ void lag_tile(const Parts<float> &P, const Mesh &m, const LagWin &win,
                                         unsigned long long *__restrict__ acc, const G4<float> *__restrict__ G,
                                         const GKD &gc, float *stage = nullptr,
                                         unsigned long long *bars = nullptr, int *err = nullptr,
                                         int *stage_fail = nullptr, unsigned btile = 0, unsigned parity = 0,
                                         uint32_t *wsh = nullptr) {
    static_assert(!PERSIST || (STAGED && FUSED), "a persistent tile is staged and fused");
    constexpr int NT = LX * LY * LZ;
    constexpr int NPT = LX * LY * LZ / THREADS;  // particles per thread
    static_assert(NPT * THREADS == LX * LY * LZ, "tile must be a multiple of the block");
    constexpr int NW = THREADS / 32;
    // Each thread takes NPT particles that follow each other along the
    // tile's slowest axis (z in 3D), so that one particle's upper corners can
    // meet the next one's lower corners in registers (see the deposit);
    // lanes of a warp take consecutive x, so loads stay coalesced.
    constexpr int NS = R == 3 ? LZ : R == 2 ? LY : LX;  // tile cells along the slowest axis
    constexpr int PL = NT / NS;                          // particles per layer of that axis
    static_assert(THREADS % PL == 0 && (THREADS / PL) * NPT == NS, "threads must cover whole layers");
    auto tidx = [](int j) { return (((int)threadIdx.x / PL) * NPT + j) * PL + (int)threadIdx.x % PL; };
    constexpr bool KEEP = STAGED && LAG_STAGE_KEEP;
    extern __shared__ __align__(16) uint32_t lag_dyn[];
    uint32_t *lag_sh = PERSIST ? wsh : KEEP ? reinterpret_cast<uint32_t *>(stage + 6 * NT) : lag_dyn;  // the window
    __shared__ int wred[6][NW];
    __shared__ int org[6];  // window origin per axis, then the extent of the box to flush
    const int cells = win.cells;
    if constexpr (KEEP && !PERSIST) {  // the window is free from the start: clear it while the copies arrive
        uint4 *z4 = reinterpret_cast<uint4 *>(lag_sh);
        for (int c = threadIdx.x; c < cells * LAG_PLANES / 4; c += THREADS) z4[c] = make_uint4(0u, 0u, 0u, 0u);
    }

    const int s = P.mshift;
    const int ntx = (1 << s) / LX, nty = R >= 2 ? (1 << s) / LY : 1, ntz = R == 3 ? (1 << s) / LZ : 1;
    const unsigned tiles = (unsigned)(ntx * nty * ntz);
    const unsigned bid = PERSIST ? btile : blockIdx.x;
    const unsigned member = bid / tiles, tile = bid % tiles;
    const int tx0 = (int)(tile % ntx) * LX;
    const int ty0 = R >= 2 ? (int)((tile / ntx) % nty) * LY : 0;
    const int tz0 = R == 3 ? (int)(tile / (ntx * nty)) * LZ : 0;
    const size_t pbase = (size_t)member << P.bshift;
    const size_t cb = (size_t)member << m.cshift;
    const int f = P.f;
    const uint32_t mask = (uint32_t)m.n - 1;
    // this member's arrays: every index below is a 32-bit offset into them
    float *dm[3];
    float *pm[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dm[k] = k < R ? P.d[k] + pbase : nullptr;
        pm[k] = k < R ? P.p[k] + pbase : nullptr;
    }
    unsigned long long *__restrict__ accm = acc + cb;

    // displacements of this thread's particles (their cells and fractions
    // are recomputed from these when depositing) and the box of their cells
    float dd[KEEP ? 1 : NPT][3];
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
#pragma unroll
    for (int j = 0; j < NPT; ++j) {
        const int t = tidx(j);
        const int lx = t % LX, ly = (t / LX) % LY, lz = t / (LX * LY);
        const int c[3] = {tx0 + lx, ty0 + ly, tz0 + lz};
        uint32_t i = (uint32_t)c[0];
        if (R >= 2) i += (uint32_t)c[1] << s;
        if (R == 3) i += (uint32_t)c[2] << (2 * s);
        float d[3];
        if constexpr (FUSED) {
            float p[3];
#pragma unroll
            for (int k = 0; k < R; ++k) {  // read once: evict-first, L1 stays for the gradients
                if constexpr (STAGED) {
                    // group j holds this thread's particle j
                    if (k == 0 && !tma_wait(bars + j, TMA_WAIT_LIMIT, parity)) {
                        atomicOr(err, 8);
                        *stage_fail = 1;
                    }
                    d[k] = stage[k * NT + t];
                    p[k] = stage[(3 + k) * NT + t];
                } else {
                    d[k] = __ldcs(dm[k] + i);
                    p[k] = __ldcs(pm[k] + i);
                }
            }
            if (gc.kick) {
                float F[3];
                const int q[3] = {c[0] * f, R >= 2 ? c[1] * f : 0, R == 3 ? c[2] * f : 0};
                gather_g4<R>(G + cb, m.shift, mask, q, d, gc.periodic, F);
                const float ck = (float)gc.ck;
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    p[k] -= F[k] * ck;
                    __stcs(pm[k] + i, p[k]);
                }
            }
            if (gc.drift) {
                const float cd = (float)gc.cd;
#pragma unroll
                for (int k = 0; k < R; ++k) {
                    d[k] += p[k] * cd;
                    __stcs(dm[k] + i, d[k]);
                    if constexpr (KEEP) stage[k * NT + t] = d[k];
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < R; ++k) d[k] = __ldg(dm[k] + i);
        }
#pragma unroll
        for (int k = 0; k < R; ++k) {
            if constexpr (!KEEP) dd[j][k] = d[k];
            int ck;
            uint32_t fk;
            quant_pos(d[k], &ck, &fk);
            const int uk = c[k] * f + ck;
            lo[k] = min(lo[k], uk);
            hi[k] = max(hi[k], uk);
        }
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        int a = __reduce_min_sync(FULL, lo[k]), b = __reduce_max_sync(FULL, hi[k]);
        if (lane == 0) {
            wred[k][wid] = a;
            wred[3 + k][wid] = b;
        }
    }
    if constexpr (STAGED) {
        __syncthreads();  // staged particles are read before the window reuses the memory
        if (*stage_fail) {
            // a copy did not arrive in time: wait (bounded again) for the
            // copies still in flight into this memory, then deposit nothing
            if (threadIdx.x == 0)
                for (int j = 0; j < NPT; ++j) tma_wait(bars + j, TMA_WAIT_LIMIT, parity);
            __syncthreads();
            return;
        }
    }
    if (!gc.deposit) return;  // a kick-only launch (the last of a run): no deposit
    if constexpr (!KEEP) {
        uint4 *z4 = reinterpret_cast<uint4 *>(lag_sh);
        for (int c = threadIdx.x; c < cells * LAG_PLANES / 4; c += THREADS) z4[c] = make_uint4(0u, 0u, 0u, 0u);
    }
    __syncthreads();
    if (threadIdx.x < R) {
        const int k = threadIdx.x;
        int a = INT_MAX, b = INT_MIN;
        for (int j = 0; j < NW; ++j) {
            a = min(a, wred[k][j]);
            b = max(b, wred[3 + k][j]);
        }
        const int W = win.w[k], ext = b - a + 2;  // corners reach hi + 1
        // the window starts at the box when the box fits (only the box is
        // flushed), else it is centred on the box (all of it is flushed)
        org[k] = ext <= W ? a : (int)(((long long)a + b + 1) >> 1) - W / 2;
        org[3 + k] = ext <= W ? ext : W;
    }
    if (threadIdx.x >= R && threadIdx.x < 3) org[3 + threadIdx.x] = 1;
    __syncthreads();

    const int o0 = org[0], o1 = R >= 2 ? org[1] : 0, o2 = R == 3 ? org[2] : 0;
    const int W0 = win.w[0], W1 = win.w[1], W2 = win.w[2], W01 = W0 * W1;
    constexpr int NB = 1 << R, HALF = NB / 2;  // corners; the upper half has the slowest axis' bit set
    // global cell of corner b of a particle in (unwrapped) cell uc
    auto corner_g = [&](const int *uc, int b) {
        uint32_t g = (uint32_t)(uc[0] + (b & 1)) & mask;
        if (R >= 2) g |= ((uint32_t)(uc[1] + ((b >> 1) & 1)) & mask) << m.shift;
        if (R == 3) g |= ((uint32_t)(uc[2] + ((b >> 2) & 1)) & mask) << (2 * m.shift);
        return g;
    };
    auto woff = [&](int b) { return (b & 1) + ((b >> 1) & 1) * W0 + ((b >> 2) & 1) * W01; };
    // adds v into window cell wc (corner b of a particle in cell uc)
    auto win_add = [&](int wc, uint32_t v, const int *uc, int b) {
        if constexpr (LAG_PLANES == 2) {
            Slot<float>::add(lag_sh, wc, v, cells);
        } else if (v) {
            // one plane: a carry out of the 32-bit cell goes to the
            // accumulator mesh directly (rare: over 2^9 particles' weight)
            const uint32_t old = atomicAdd(lag_sh + wc, v);
            if (old + v < old) atomicAdd(accm + corner_g(uc, b), 1ull << 32);
        }
    };
    // the upper corners of this thread's previous particle, held back while
    // they may coincide with the next particle's lower corners (the next
    // particle one cell further along the slowest axis): their integer
    // weights are then added in registers before one window add
    bool pend = false;
    int pu[3] = {0, 0, 0}, pwc = 0;
    uint32_t pw[HALF];
#pragma unroll
    for (int j = 0; j < NPT; ++j) {
        // cells (unwrapped) and 21-bit fractions of the deposit position
        int u[3] = {0, 0, 0};
        uint32_t fr[3];
        {
            const int t = tidx(j);
            const int c[3] = {tx0 + t % LX, ty0 + (t / LX) % LY, tz0 + t / (LX * LY)};
#pragma unroll
            for (int k = 0; k < R; ++k) {
                int ck;
                quant_pos(KEEP ? stage[k * NT + t] : dd[j][k], &ck, &fr[k]);
                u[k] = c[k] * f + ck;
            }
        }
        float f0 = (float)fr[0] * 0x1p-21f;
        float wx[2] = {1.0f - f0, f0}, wy[2] = {1.0f, 1.0f}, wz[2] = {1.0f, 1.0f};
        if (R >= 2) {
            float f1 = (float)fr[1] * 0x1p-21f;
            wy[0] = 1.0f - f1;
            wy[1] = f1;
        }
        if (R == 3) {
            float f2 = (float)fr[2] * 0x1p-21f;
            wz[0] = 1.0f - f2;
            wz[1] = f2;
        }
        uint32_t v[NB];
#pragma unroll
        for (int b = 0; b < NB; ++b) v[b] = quant_w(wx[b & 1] * wy[(b >> 1) & 1] * wz[(b >> 2) & 1]);
        const int l0 = u[0] - o0, l1 = R >= 2 ? u[1] - o1 : 0, l2 = R == 3 ? u[2] - o2 : 0;
        const bool inside = l0 >= 0 && l0 + 1 < W0 && (R < 2 || (l1 >= 0 && l1 + 1 < W1)) &&
                            (R < 3 || (l2 >= 0 && l2 + 1 < W2));
        if (pend) {
            bool meet = inside && u[R - 1] == pu[R - 1] + 1;
#pragma unroll
            for (int k = 0; k < R - 1; ++k) meet = meet && u[k] == pu[k];
            if (meet) {
#pragma unroll
                for (int h = 0; h < HALF; ++h) v[h] += pw[h];  // <= 2^24: no overflow
            } else {
#pragma unroll
                for (int h = 0; h < HALF; ++h) win_add(pwc + woff(HALF + h), pw[h], pu, HALF + h);
            }
            pend = false;
        }
        if (inside) {
            const int base = (l2 * W1 + l1) * W0 + l0;
#pragma unroll
            for (int h = 0; h < HALF; ++h) win_add(base + woff(h), v[h], u, h);
            if (j + 1 < NPT) {
                pend = true;
                pwc = base;
#pragma unroll
                for (int k = 0; k < 3; ++k) pu[k] = u[k];
#pragma unroll
                for (int h = 0; h < HALF; ++h) pw[h] = v[HALF + h];
            } else {
#pragma unroll
                for (int h = 0; h < HALF; ++h) win_add(base + woff(HALF + h), v[HALF + h], u, HALF + h);
            }
        } else {
#pragma unroll
            for (int b = 0; b < NB; ++b)
                if (v[b]) atomicAdd(accm + corner_g(u, b), (unsigned long long)v[b]);
        }
    }
    __syncthreads();

    // flush the box E0 x E1 x E2 at the window's origin: thread t visits box
    // cells t, t + THREADS, ...; the coordinates advance incrementally (no
    // divisions in the loop)
    const int E0 = org[3], E1 = org[4], E2 = org[5];
    const int ecells = E0 * E1 * E2;
    int l0 = (int)threadIdx.x % E0, l1 = ((int)threadIdx.x / E0) % E1, l2 = (int)threadIdx.x / (E0 * E1);
    const int s0 = THREADS % E0, s1 = (THREADS / E0) % E1, s2 = THREADS / (E0 * E1);
    for (int c = threadIdx.x; c < ecells; c += THREADS) {
        const int wc = (l2 * W1 + l1) * W0 + l0;
        uint32_t a = lag_sh[wc], b = LAG_PLANES == 2 ? lag_sh[cells + wc] : 0u;
        if constexpr (PERSIST) {  // leave the window clear for the next tile
            lag_sh[wc] = 0u;
            if (LAG_PLANES == 2) lag_sh[cells + wc] = 0u;
        }
        if (a | b) {
            uint32_t g = (uint32_t)(o0 + l0) & mask;
            if (R >= 2) g |= ((uint32_t)(o1 + l1) & mask) << m.shift;
            if (R == 3) g |= ((uint32_t)(o2 + l2) & mask) << (2 * m.shift);
            atomicAdd(accm + g, ((unsigned long long)b << 32) | a);
        }
        l0 += s0;
        l1 += s1;
        l2 += s2;
        if (l0 >= E0) {
            l0 -= E0;
            ++l1;
        }
        if (l1 >= E1) {
            l1 -= E1;
            ++l2;
        }
    }
}

template <int R, int LX, int LY, int LZ, int THREADS>
__global__ void __launch_bounds__(THREADS)
    k_deposit_lag(Parts<float> P, Mesh m, LagWin win, unsigned long long *__restrict__ acc) {
    lag_tile<R, LX, LY, LZ, THREADS, false>(P, m, win, acc, nullptr, GKD{});
}

// Gather + kick + drift of k_gkd (FD4 gradient) fused with the Lagrangian
// deposit of the drifted positions into the accumulator mesh.
template <int R, int LX, int LY, int LZ, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
    k_gkd_lag(Parts<float> P, Mesh m, const G4<float> *__restrict__ G, GKD gc, LagWin win,
              unsigned long long *__restrict__ acc) {
    lag_tile<R, LX, LY, LZ, THREADS, true>(P, m, win, acc, G, gc);
}

// ------------------------------------------- TMA staging of a 3D tile --
//
// The six particle arrays of a 3D lattice tile (d[0..2], p[0..2], LX x LY x
// LZ floats each, in tile order) come from tensor maps over the (N, N,
// N*batch) arrays, one z-plane per bulk tensor copy, in NPT groups: group j
// holds every thread's particle j (the planes s NPT + j).
// Thread 0 issues the bulk tensor copies of all groups at once, each group
// completing its own mbarrier, and every thread waits for group j just
// before it needs particle j, so the first particles are computed while the
// rest arrive. Waits are bounded: a wait that runs out after TMA_WAIT_LIMIT
// polls sets bit 3 (value 8) of the error word (CONAN_ERR_TIMEOUT on the
// host) and the tile, after one more bounded wait for its copies in flight,
// deposits nothing. No multicast: every copy reads this GPU's own memory into
// this CTA.
struct TileMaps {
    CUtensorMap a[6];  // d0, d1, d2, p0, p1, p2; box LX x LY x 1
};

__device__ inline uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Waits for the completion of the phase of parity `parity` of mbarrier
// `bar`, at most `limit` polls; false when the wait ran out.
__device__ inline bool tma_wait(unsigned long long *bar, unsigned limit, unsigned parity) {
    const uint32_t b = smem_addr(bar);
    uint32_t done = 0;
    for (unsigned it = 0; it < limit && !done; ++it)
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b), "r"(parity)
            : "memory");
    return done != 0;
}

template <int R, int LX, int LY, int LZ, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
    k_gkd_lag_tma(Parts<float> P, Mesh m, const G4<float> *__restrict__ G, GKD gc, LagWin win,
                  unsigned long long *__restrict__ acc, const __grid_constant__ TileMaps maps, int *err) {
    static_assert(R == 3, "the staged tile is three-dimensional");
    constexpr int NT = LX * LY * LZ, NPT = NT / THREADS, GP = THREADS / (LX * LY);
    static_assert(GP * NPT == LZ && GP * LX * LY == THREADS, "a group of z-planes holds one particle per thread");
    extern __shared__ __align__(16) uint32_t lag_sh[];
    __shared__ __align__(8) unsigned long long bars[NPT];
    __shared__ int stage_fail;
    // bulk tensor copies land on 128-byte boundaries (the launch adds 128 bytes)
    float *stage = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(lag_sh) + 127) & ~(uintptr_t)127);
    const int s = P.mshift;
    const int ntx = (1 << s) / LX, nty = (1 << s) / LY, ntz = (1 << s) / LZ;
    const unsigned tiles = (unsigned)(ntx * nty * ntz);
    const unsigned member = blockIdx.x / tiles, tile = blockIdx.x % tiles;
    const int x0 = (int)(tile % ntx) * LX, y0 = (int)((tile / ntx) % nty) * LY;
    const int z0 = (int)(tile / (ntx * nty)) * LZ + (int)(member << s);
    if (threadIdx.x == 0) {
        stage_fail = 0;
#pragma unroll
        for (int j = 0; j < NPT; ++j) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bars + j)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int j = 0; j < NPT; ++j) {
            const uint32_t b = smem_addr(bars + j);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(6u * THREADS * 4u)
                         : "memory");
            // group j: the planes s NPT + j, one box (LX x LY x 1) each
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int q = 0; q < GP; ++q) {
                    const int lz = q * NPT + j;
                    asm volatile(
                        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(stage + a * NT + lz * LX * LY)),
                        "l"(reinterpret_cast<uint64_t>(&maps.a[a])), "r"(x0), "r"(y0), "r"(z0 + lz), "r"(b)
                        : "memory");
                }
        }
    }
    lag_tile<R, LX, LY, LZ, THREADS, true, true>(P, m, win, acc, G, gc, stage, bars, err, &stage_fail);
}

// Persistent form of the staged fused launch: a CTA loops over tiles t,
// t + gridDim.x, ... and, while it works on one tile, the bulk tensor copies
// of its next tile land in a second staging buffer, so the particle stream
// never waits for a tile's start. Two buffers of the six arrays (one
// mbarrier per particle group and buffer; use k of a buffer completes phase
// k), then the window, which is cleared once here and kept clear by the
// flush of every tile. Waits are bounded as in k_gkd_lag_tma; after one runs
// out the CTA waits (bounded) for its copies in flight and stops.
template <int R, int LX, int LY, int LZ, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
    k_gkd_lag_pers(Parts<float> P, Mesh m, const G4<float> *__restrict__ G, GKD gc, LagWin win,
                   unsigned long long *__restrict__ acc, const __grid_constant__ TileMaps maps, int *err,
                   unsigned ntiles) {
    static_assert(R == 3, "the staged tile is three-dimensional");
    constexpr int NT = LX * LY * LZ, NPT = NT / THREADS, GP = THREADS / (LX * LY);
    static_assert(GP * NPT == LZ && GP * LX * LY == THREADS, "a group of z-planes holds one particle per thread");
    extern __shared__ __align__(16) uint32_t lag_dyn[];
    __shared__ __align__(8) unsigned long long bars[2][NPT];
    __shared__ int stage_fail;
    float *stage0 = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(lag_dyn) + 127) & ~(uintptr_t)127);
    float *stage1 = stage0 + 6 * NT;
    uint32_t *wsh = reinterpret_cast<uint32_t *>(stage1 + 6 * NT);
    const int s = P.mshift;
    const int ntx = (1 << s) / LX, nty = (1 << s) / LY, ntz = (1 << s) / LZ;
    const unsigned tiles = (unsigned)(ntx * nty * ntz);
    if (threadIdx.x == 0) {
        stage_fail = 0;
        for (int q = 0; q < 2 * NPT; ++q)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bars[0][0] + q)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    uint4 *z4 = reinterpret_cast<uint4 *>(wsh);
    for (int c = threadIdx.x; c < win.cells * LAG_PLANES / 4; c += THREADS) z4[c] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    // thread 0: the copies of tile t into buffer q (group j: the planes
    // g NPT + j of the tile, one box LX x LY x 1 each)
    auto issue = [&](unsigned t, int q) {
        const unsigned member = t / tiles, tile = t % tiles;
        const int x0 = (int)(tile % ntx) * LX, y0 = (int)((tile / ntx) % nty) * LY;
        const int z0 = (int)(tile / (ntx * nty)) * LZ + (int)(member << s);
        float *st = q ? stage1 : stage0;
        for (int j = 0; j < NPT; ++j) {
            const uint32_t b = smem_addr(&bars[q][j]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(6u * THREADS * 4u)
                         : "memory");
#pragma unroll
            for (int a = 0; a < 6; ++a)
#pragma unroll
                for (int g = 0; g < GP; ++g) {
                    const int lz = g * NPT + j;
                    asm volatile(
                        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(st + a * NT + lz * LX * LY)),
                        "l"(reinterpret_cast<uint64_t>(&maps.a[a])), "r"(x0), "r"(y0), "r"(z0 + lz), "r"(b)
                        : "memory");
                }
        }
    };
    unsigned t = blockIdx.x;
    if (threadIdx.x == 0 && t < ntiles) issue(t, 0);
    for (unsigned it = 0; t < ntiles; t += gridDim.x, ++it) {
        const int b = (int)(it & 1);
        // the other buffer was last read by the previous tile's deposit,
        // which every thread finished before that tile's flush
        if (threadIdx.x == 0 && t + gridDim.x < ntiles) issue(t + gridDim.x, b ^ 1);
        lag_tile<R, LX, LY, LZ, THREADS, true, true, true>(P, m, win, acc, G, gc, b ? stage1 : stage0, bars[b], err,
                                                            &stage_fail, t, (it >> 1) & 1, wsh);
        if (stage_fail) {  // set before a barrier inside lag_tile: the same for every thread
            if (threadIdx.x == 0 && t + gridDim.x < ntiles)
                for (int j = 0; j < NPT; ++j) tma_wait(&bars[b ^ 1][j], TMA_WAIT_LIMIT, ((it + 1) >> 1) & 1);
            __syncthreads();
            return;
        }
    }
}

// Density contrast from the integer accumulator (units of 2^-23 particle
// weights): out = sum 2^-23 mass - 1, as the sorted deposit. The caller
// clears the accumulator afterwards (a plain memset streams faster than
// zero stores mixed into this read stream).
template <typename T>
__global__ void __launch_bounds__(256) k_acc_mesh(unsigned long long *__restrict__ acc, T *__restrict__ out,
                                                  size_t n, double scale) {
    const size_t i = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
    if (i + 3 < n) {  // n is a power of two >= 4 except for tiny meshes
        ulonglong2 a = *reinterpret_cast<const ulonglong2 *>(acc + i);
        ulonglong2 b = *reinterpret_cast<const ulonglong2 *>(acc + i + 2);
        const double k = 0x1p-23 * scale;
        T v0 = (T)((double)a.x * k - 1.0), v1 = (T)((double)a.y * k - 1.0);
        T v2 = (T)((double)b.x * k - 1.0), v3 = (T)((double)b.y * k - 1.0);
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4 *>(out + i) = make_float4(v0, v1, v2, v3);
        } else {
            out[i] = v0;
            out[i + 1] = v1;
            out[i + 2] = v2;
            out[i + 3] = v3;
        }
    } else {
        for (size_t j = i; j < n; ++j) out[j] = (T)((double)acc[j] * (0x1p-23 * scale) - 1.0);
    }
}

// ------------------------------------------------------------ init/io --

// Zel'dovich start (Zeldovich<R>, src/run/nbody.hh:26-51): u = FD4(phi_m)
// on the mass mesh; d = cdz u, p = cpz u with cdz = -a_pos/(res_m res_f),
// cpz = -a_mom/(res_m res_f).
template <typename T, int R>
__global__ void k_zeldovich(Parts<T> P, const T *__restrict__ phim, Mesh mm, double cdz, double cpz) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    int c[3];
#pragma unroll
    for (int k = 0; k < R; ++k) c[k] = (int)((i >> (k * mm.shift)) & (size_t)(mm.n - 1));
#pragma unroll
    for (int k = 0; k < R; ++k) {
        T u = fd4<T, R>(phim + member_cells(mm, i >> P.bshift), c, k, mm.shift, mm.n - 1);
        P.d[k][i] = u * (T)cdz;
        P.p[k][i] = u * (T)cpz;
    }
}

// Absolute positions / momenta (AoS doubles) of particles i0 .. i0+cnt-1
// from the lattice state, written from X[0], Pm[0] on (either may be null).
template <typename T, int R>
__global__ void k_export(Parts<T> P, double res, size_t i0, size_t cnt, double *__restrict__ X,
                         double *__restrict__ Pm) {
    const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cnt) return;
    const size_t i = i0 + j;
    int q[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        if (X) X[j * R + k] = ((double)q[k] + (double)P.d[k][i]) * res;
        if (Pm) Pm[j * R + k] = (double)P.p[k][i] * res;
    }
}

// The inverse of k_export for particles i0 .. i0+cnt-1.
template <typename T, int R>
__global__ void k_import(Parts<T> P, double res, size_t i0, size_t cnt, const double *__restrict__ X,
                         const double *__restrict__ Pm) {
    const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cnt) return;
    const size_t i = i0 + j;
    int q[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        P.d[k][i] = (T)(X[j * R + k] / res - (double)q[k]);
        P.p[k][i] = (T)(Pm[j * R + k] / res);
    }
}

template <typename S, typename D>
__global__ void k_convert(const S *__restrict__ in, D *__restrict__ out, size_t n, double scale,
                          double shift) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (D)((double)in[i] * scale + shift);
}

// ------------------------------------------------------ power spectrum --

// Per-block partial sums of |delta_hat|^2, |k| and mode count per shell
// floor(|n| + 1/2). Each warp takes a 32-wide run of one half-spectrum row,
// where the shell index is nondecreasing, and sums runs of equal shells with
// a fixed shuffle pattern; warps and blocks are combined in fixed order.
template <typename T>
__global__ void k_pk_partial(const typename Cplx<T>::type *__restrict__ spec, Mesh m, int nbins,
                             double *__restrict__ part) {
    extern __shared__ double pk_sh[];  // [warps][3][nbins]
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double *mine = pk_sh + (size_t)w * 3 * nbins;
    for (int j = lane; j < 3 * nbins; j += 32) mine[j] = 0;
    __syncwarp();
    const int segs = (m.nh + 31) / 32;
    const size_t rows = m.spec / m.nh;
    const long long ntask = (long long)rows * segs;
    for (long long t = (long long)blockIdx.x * nw + w; t < ntask; t += (long long)gridDim.x * nw) {
        size_t row = (size_t)(t / segs);
        int kx = (int)(t % segs) * 32 + lane;
        bool act = kx < m.nh;
        size_t e = row * m.nh + (act ? kx : 0);
        int kv[3];
        long long k2 = spec_k2(e, m, kv);
        double nn = sqrt((double)k2);
        int bin = act ? (int)floor(nn + 0.5) : nbins;
        if (bin >= nbins) bin = nbins;
        double wt = act ? spec_weight(kx, m.n) : 0.0;
        auto z = spec[e];
        double v[3] = {wt * ((double)z.x * z.x + (double)z.y * z.y), wt * nn, wt};
        bool leader;
        (void)leader;
        // inclusive segmented scan over runs of equal bins
        int prev = __shfl_up_sync(FULL, bin, 1);
        bool head = lane == 0 || bin != prev;
        unsigned heads = __ballot_sync(FULL, head);
        int start = 31 - __clz(heads & (FULL >> (31 - lane)));
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                double u = __shfl_up_sync(FULL, v[q], o);
                if (lane - o >= start) v[q] += u;
            }
        }
        int next = __shfl_down_sync(FULL, bin, 1);
        bool tail = lane == 31 || next != bin;
        if (tail && bin < nbins) {
            mine[bin] += v[0];
            mine[nbins + bin] += v[1];
            mine[2 * nbins + bin] += v[2];
        }
        __syncwarp();
    }
    __syncthreads();
    for (int j = threadIdx.x; j < 3 * nbins; j += blockDim.x) {
        double s = 0;
        for (int q = 0; q < nw; ++q) s += pk_sh[(size_t)q * 3 * nbins + j];
        part[(size_t)blockIdx.x * 3 * nbins + j] = s;
    }
}

}  // namespace conan
