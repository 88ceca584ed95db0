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
// cell id followed by a warp-segmented reduction:
//   rank   : cell id of every particle (integer, periodic wrap), rank within
//            its cell from an integer counter (fused into the drift),
//   scan   : exclusive prefix of the per-cell counts -> cell offsets,
//   scatter: the particle's cell fractions written at offset + rank,
//   reduce : each warp walks a 32-cell row of cells in sorted order; the
//            2^R corner weights of each particle are quantised to integers
//            and summed per cell with redux.sync over runs of lanes holding
//            the same cell, then combined with the neighbouring rows and
//            planes in registers. All sums are integer, so the density is
//            bit-identical from run to run whatever order the sort produced
//            inside a cell; no floating-point atomics are used.
#pragma once

#include "common.cuh"

namespace conan {

constexpr unsigned FULL = 0xffffffffu;

template <typename T> struct Parts {
    T *d[3];
    T *p[3];
    size_t np;
    int mshift;  // log2(N_m)
    int f;       // force cells per lattice spacing
};

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
    rank[i] = atomicAdd(count + c, 1u);
}

// ------------------------------------------------------------ scan --

constexpr int SCAN_T = 256, SCAN_V = 16, SCAN_CHUNK = SCAN_T * SCAN_V;

static __global__ void __launch_bounds__(SCAN_T) k_scan_partial(const uint32_t *__restrict__ count,
                                                         size_t n, uint32_t *__restrict__ bsum) {
    size_t base = (size_t)blockIdx.x * SCAN_CHUNK + (size_t)threadIdx.x * SCAN_V;
    uint32_t s = 0;
    if (base + SCAN_V <= n) {
        const uint4 *v = reinterpret_cast<const uint4 *>(count + base);
#pragma unroll
        for (int j = 0; j < SCAN_V / 4; ++j) {
            uint4 x = v[j];
            s += x.x + x.y + x.z + x.w;
        }
    } else {
        for (size_t j = base; j < n; ++j) s += count[j];
    }
    s = block_sum<uint32_t>(s);
    if (threadIdx.x == 0) bsum[blockIdx.x] = s;
}

// Single-block exclusive scan of the block sums (nb <= 1024 * 1024).
static __global__ void __launch_bounds__(1024) k_scan_blocks(uint32_t *bsum, int nb) {
    __shared__ uint32_t wsum[32];
    int per = (nb + 1023) / 1024;
    int beg = threadIdx.x * per, end = min(beg + per, nb);
    uint32_t s = 0;
    for (int j = beg; j < end; ++j) s += bsum[j];
    // block exclusive scan of s
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = s;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(FULL, inc, o);
        if (lane >= o) inc += v;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t v = wsum[lane];
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t u = __shfl_up_sync(FULL, v, o);
            if (lane >= o) v += u;
        }
        wsum[lane] = v;
    }
    __syncthreads();
    uint32_t run = inc - s + (w > 0 ? wsum[w - 1] : 0u);
    for (int j = beg; j < end; ++j) {
        uint32_t c = bsum[j];
        bsum[j] = run;
        run += c;
    }
}

// Exclusive offsets of every cell (off[n] = total) and counts reset to 0.
static __global__ void __launch_bounds__(SCAN_T) k_scan_final(uint32_t *__restrict__ count, size_t n,
                                                       const uint32_t *__restrict__ bsum,
                                                       uint32_t *__restrict__ off) {
    __shared__ uint32_t wsum[SCAN_T / 32];
    size_t base = (size_t)blockIdx.x * SCAN_CHUNK + (size_t)threadIdx.x * SCAN_V;
    uint32_t v[SCAN_V];
    bool full = base + SCAN_V <= n;
    if (full) {
        uint4 *p = reinterpret_cast<uint4 *>(count + base);
#pragma unroll
        for (int j = 0; j < SCAN_V / 4; ++j) {
            uint4 x = p[j];
            v[4 * j] = x.x;
            v[4 * j + 1] = x.y;
            v[4 * j + 2] = x.z;
            v[4 * j + 3] = x.w;
            p[j] = make_uint4(0, 0, 0, 0);
        }
    } else {
#pragma unroll
        for (int j = 0; j < SCAN_V; ++j) {
            v[j] = (base + j < n) ? count[base + j] : 0u;
            if (base + j < n) count[base + j] = 0u;
        }
    }
    uint32_t s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_V; ++j) s += v[j];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = s;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t u = __shfl_up_sync(FULL, inc, o);
        if (lane >= o) inc += u;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    uint32_t wpre = 0;
    for (int j = 0; j < w; ++j) wpre += wsum[j];
    uint32_t run = bsum[blockIdx.x] + wpre + inc - s;
    if (full) {
        uint4 *o = reinterpret_cast<uint4 *>(off + base);
#pragma unroll
        for (int j = 0; j < SCAN_V / 4; ++j) {
            uint4 x;
            x.x = run; run += v[4 * j];
            x.y = run; run += v[4 * j + 1];
            x.z = run; run += v[4 * j + 2];
            x.w = run; run += v[4 * j + 3];
            o[j] = x;
        }
    } else {
        for (int j = 0; j < SCAN_V; ++j) {
            if (base + j < n) off[base + j] = run;
            run += v[j];
        }
    }
    if (base < n && base + SCAN_V >= n) off[n] = run;
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
        uint32_t dst = off[c] + rank[i];
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
        uint32_t dst = off[c] + rank[i];
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

// Lanes of the run of equal `cell` values containing this lane (cells are
// nondecreasing across the warp), and whether this lane leads it.
__device__ inline unsigned run_mask(int cell, int lane, bool *leader) {
    int prev = __shfl_up_sync(FULL, cell, 1);
    bool head = lane == 0 || cell != prev;
    unsigned heads = __ballot_sync(FULL, head);
    unsigned upto = FULL >> (31 - lane);
    int start = 31 - __clz(heads & upto);
    unsigned above = lane == 31 ? 0u : (heads & (FULL << (lane + 1)));
    int end = above ? (__ffs(above) - 2) : 31;
    *leader = lane == start;
    unsigned hi = end == 31 ? FULL : ((1u << (end + 1)) - 1u);
    return hi & (FULL << start);
}

// Segmented integer sum of the quantised weight over a run of lanes.
__device__ inline unsigned long long run_sum(unsigned mask, uint32_t q) {
    return __reduce_add_sync(mask, q);
}
__device__ inline unsigned long long run_sum(unsigned mask, unsigned long long q) {
    uint32_t hi = (uint32_t)(q >> 26), lo = (uint32_t)(q & 0x3FFFFFFull);
    unsigned long long sh = __reduce_add_sync(mask, hi), sl = __reduce_add_sync(mask, lo);
    return (sh << 26) + sl;
}
__device__ inline void acc_add(unsigned long long &a, unsigned long long v) { a += v; }
__device__ inline void acc_add(U128 &a, unsigned long long v) { a = a + U128{v, 0ull}; }

// One warp deposits a strip of 32 cells along axis 0 for YW rows (R >= 2) and
// ZC planes (R == 3): out[c] = mass * sum of corner weights - 1.
// Requires n % 32 == 0, n % YW == 0, n % ZC == 0.
template <typename T, int R, int YW, int ZC, int WPB>
__global__ void __launch_bounds__(WPB * 32)
    k_deposit(const uint32_t *__restrict__ off, const typename Pay<T>::elem *__restrict__ pay,
              T *__restrict__ out, Mesh m, double scale, uint32_t np, int *__restrict__ err) {
    typedef typename Acc<T>::type A;
    constexpr int C = 1 << R;
    __shared__ A slots[WPB][34][C];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int n = m.n, mask = n - 1;
    const int nxs = n >> 5, nys = R >= 2 ? n / YW : 1, nzs = R == 3 ? n / ZC : 1;
    long long task = (long long)blockIdx.x * WPB + w;
    if (task >= (long long)nxs * nys * nzs) return;
    const int xs = (int)(task % nxs);
    const int ys = (int)((task / nxs) % nys);
    const int zs = (int)(task / ((long long)nxs * nys));
    const int x0 = xs * 32, y0 = ys * YW, z0 = zs * ZC;
    const int hx = (x0 - 1) & mask;

    for (int j = lane; j < 34 * C; j += 32) (&slots[w][0][0])[j] = Acc<T>::zero();
    __syncwarp();

    A plane[YW > 0 ? YW : 1];
#pragma unroll
    for (int y = 0; y < (YW > 0 ? YW : 1); ++y) plane[y] = Acc<T>::zero();

    const int zlo = R == 3 ? -1 : 0, zhi = R == 3 ? ZC : 1;
    for (int zz = zlo; zz < zhi; ++zz) {
        const int z = (z0 + zz) & mask;
        A rowc[2] = {Acc<T>::zero(), Acc<T>::zero()};
#pragma unroll
        for (int yi = 0; yi < (R >= 2 ? YW + 1 : 1); ++yi) {
            const int yy = R >= 2 ? yi - 1 : 0;
            const int y = (y0 + yy) & mask;
            size_t rb = 0;
            if (R == 2) rb = (size_t)y << m.shift;
            if (R == 3) rb = ((size_t)z << (2 * m.shift)) | ((size_t)y << m.shift);

            // Cell ranges of this row: halo cell x0-1 (logical cell 0) and
            // cells x0..x0+31 (logical cells 1..32).
            uint32_t e = __ldg(off + rb + x0 + lane + 1);
            uint32_t b0 = __ldg(off + rb + x0);
            uint32_t hb = __ldg(off + rb + hx), he = __ldg(off + rb + hx + 1);
            uint32_t hcount = he - hb;
            uint32_t Bv = hcount + (e - b0);
            uint32_t total = __shfl_sync(FULL, Bv, 31);
            // Offsets are monotone by construction; never walk a corrupt range.
            if (__any_sync(FULL, e < b0 || he < hb) || total > np) {
                if (lane == 0) atomicOr(err, 2);
                total = 0;
            }

            for (uint32_t base = 0; base < total; base += 32) {
                uint32_t j = base + lane;
                bool active = j < total;
                // Binary search over the 32 cell ends held by the lanes (all
                // lanes take part in every shuffle).
                int pos = 0;
#pragma unroll
                for (int step = 16; step >= 1; step >>= 1) {
                    uint32_t v = __shfl_sync(FULL, Bv, pos + step - 1);
                    if (v <= j) pos += step;
                }
                int cell = j < hcount ? 0 : 1 + pos;
                uint32_t src = j < hcount ? hb + j : b0 + (j - hcount);
                if (!active) cell = 33;
                if (active && src >= np) {  // corrupt offsets: flag, skip
                    atomicOr(err, 1);
                    active = false;
                    cell = 33;
                }
                T fr[3] = {T(0), T(0), T(0)};
                if (active) load_frac<T, R>(pay, src, fr);
                bool leader;
                unsigned rm = run_mask(cell, lane, &leader);
#pragma unroll
                for (int b = 0; b < C; ++b) {
                    auto q = Acc<T>::quant(corner_weight<T, R>(fr, b));
                    if (!active) q = 0;
                    unsigned long long s = run_sum(rm, q);
                    if (leader) acc_add(slots[w][cell][b], s);
                }
                __syncwarp();
            }

            // Combine the row: bx via the neighbouring slot, by via the
            // previous row (rowc), bz via the previous plane (plane[]).
            A t[2][2];
#pragma unroll
            for (int by = 0; by < 2; ++by)
#pragma unroll
                for (int bz = 0; bz < 2; ++bz) {
                    t[by][bz] = Acc<T>::zero();
                    if ((by && R < 2) || (bz && R < 3)) continue;
                    int b = 2 * by + 4 * bz;
                    t[by][bz] = slots[w][lane + 1][b] + slots[w][lane][b + 1];
                }
            __syncwarp();
            for (int j = lane; j < 34 * C; j += 32) (&slots[w][0][0])[j] = Acc<T>::zero();
            __syncwarp();

            A o0, o1;
            if (R >= 2) {
                o0 = t[0][0] + rowc[0];
                o1 = t[0][1] + rowc[1];
                rowc[0] = t[1][0];
                rowc[1] = t[1][1];
            } else {
                o0 = t[0][0];
                o1 = Acc<T>::zero();
            }
            if (yy < 0) continue;
            A tot = o0;
            if (R == 3) {
                tot = o0 + plane[yy];
                plane[yy] = o1;
            }
            if (zz < 0) continue;
            out[rb + x0 + lane] = (T)(Acc<T>::value(tot) * scale - 1.0);
        }
    }
}

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
template <typename T>
__global__ void k_green(typename Cplx<T>::type *__restrict__ spec, Mesh m, T gs) {
    size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= m.spec) return;
    int kv[3];
    long long k2 = spec_k2(e, m, kv);
    T g = k2 > 0 ? gs / (T)k2 : T(0);
    auto z = spec[e];
    z.x *= g;
    z.y *= g;
    spec[e] = z;
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

// CIC-interpolated force of particle i: sum over corners of weight times
// the gradient (FD4 of phi, or the spectral gradient meshes g[k]).
template <typename T, int R, bool SPECTRAL>
__device__ inline void gather_force(const Parts<T> &P, const Mesh &m, size_t i, const T *phi,
                                    const T *const *g, bool periodic, const T *d, T *F) {
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
#pragma unroll
    for (int b = 0; b < (1 << R); ++b) {
        T z = 1;
        int c[3];
#pragma unroll
        for (int k = 0; k < R; ++k) {
            int bk = (b >> k) & 1;
            z *= bk ? a1[k] : a0[k];
            c[k] = (o[k] + bk) & mask;
        }
        if constexpr (SPECTRAL) {
            size_t ci = 0;
#pragma unroll
            for (int k = R - 1; k >= 0; --k) ci = (ci << m.shift) | (size_t)c[k];
#pragma unroll
            for (int k = 0; k < R; ++k) F[k] += __ldg(g[k] + ci) * z;
        } else {
#pragma unroll
            for (int k = 0; k < R; ++k) F[k] += fd4<T, R>(phi, c, k, m.shift, mask) * z;
        }
    }
}

struct GKD {
    double ck;  // kick: p -= F ck (0 disables)
    double cd;  // drift: d += p cd (after the kick)
    int kick, drift, rank, periodic;
};

// Fused leapfrog update of particle i: the kick of Gravity::kick
// (src/run/nbody.hh:112-117), then the next step's drift (Gravity::drift,
// src/run/nbody.hh:122-130), then the counting-sort rank of the new cell.
template <typename T, int R, bool SPECTRAL>
__global__ void __launch_bounds__(256)
    k_gkd(Parts<T> P, Mesh m, const T *__restrict__ phi, const T *__restrict__ g0,
          const T *__restrict__ g1, const T *__restrict__ g2, GKD c, uint32_t *__restrict__ count,
          uint32_t *__restrict__ rank) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
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
        gather_force<T, R, SPECTRAL>(P, m, i, phi, g, c.periodic, d, F);
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
    if (c.rank) rank[i] = atomicAdd(count + deposit_cell<T, R>(P, m, i), 1u);
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
        T u = fd4<T, R>(phim, c, k, mm.shift, mm.n - 1);
        P.d[k][i] = u * (T)cdz;
        P.p[k][i] = u * (T)cpz;
    }
}

// Absolute positions / momenta (AoS doubles) from the lattice state.
template <typename T, int R>
__global__ void k_export(Parts<T> P, double res, double *__restrict__ X, double *__restrict__ Pm) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    int q[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        if (X) X[i * R + k] = ((double)q[k] + (double)P.d[k][i]) * res;
        if (Pm) Pm[i * R + k] = (double)P.p[k][i] * res;
    }
}

template <typename T, int R>
__global__ void k_import(Parts<T> P, double res, const double *__restrict__ X,
                         const double *__restrict__ Pm) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.np) return;
    int q[3];
    lattice<T, R>(P, i, q);
#pragma unroll
    for (int k = 0; k < R; ++k) {
        P.d[k][i] = (T)(X[i * R + k] / res - (double)q[k]);
        P.p[k][i] = (T)(Pm[i * R + k] / res);
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
