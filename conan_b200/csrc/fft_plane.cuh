// fft_plane.cuh -- the x and y directions of the Poisson solve's 3D transform
// for one z plane per thread-block cluster, exchanging through distributed
// shared memory.
//
// cuFFT's 2D R2C over every z plane (and the conversion of the integer
// deposit into the density before it, and its 2D C2R after the z pass) moves
// each plane through HBM several times. Here one cluster of C CTAs owns one
// z plane of one member, each CTA KC of its kx columns (C = n / (2 KC)):
//
//   forward (k_plane_fwd): CTA r reads rows y in [r n/C, (r + 1) n/C) of the
//   integer accumulator, converts them to the density contrast exactly as
//   k_acc_mesh does, and each warp transforms its rows along x (a real FFT
//   of n points as a complex FFT of n/2 points plus the usual split,
//   Numerical Recipes section 12.3); the n/2 + 1 outputs of a row go
//   straight into the shared memory of the CTA that owns their kx columns
//   (CTA r' owns kx in [KC r', KC (r' + 1)); the DC and Nyquist columns, both
//   real per row, share column 0 of CTA 0 as DC + i Nyquist). After a
//   cluster barrier every CTA transforms its KC columns along y (n points)
//   and writes them to the half spectrum (z, ky, kx), the layout of cuFFT's
//   plane transforms that the z pass reads; CTA 0 separates DC and Nyquist.
//
//   inverse (k_plane_inv): the same steps backwards. CTA r reads its KC
//   columns of the plane (DC + i Nyquist packed again in column 0 of CTA
//   0), transforms them along y, and after a cluster barrier each warp
//   gathers whole rows of its CTA's range from the CTAs' shared memory,
//   runs the complex-to-real x transform and writes the potential.
//
// Both are unnormalised, as cuFFT's R2C and C2R, so the Green's function
// factor of the z pass is unchanged. The FFTs are the Stockham formulation
// of fft_z.cuh (same stage formula, radix-2/4/8 butterflies, twiddle table
// exp(-2 pi i k / n) and powers by recurrence): a warp-private one for the n/2
// points of an x row, a CTA-wide one over the KC lines for y.
//
// HBM traffic per plane: forward 8 n^2 bytes of accumulator read, 4 n (n + 2)
// bytes of spectrum written; inverse 4 n (n + 2) read, 4 n^2 written. The
// path it replaces moved the density (8 n^2 read, 4 n^2 written), then
// cuFFT's planes (at least 4 n^2 + 4 n (n + 2) each way).
#pragma once

#include <cooperative_groups.h>

#include "fft_z.cuh"

namespace conan {

// Sizes of the plane pass for an n-point plane with KC kx columns per CTA:
// clusters of n / (2 KC) CTAs of 512 threads, each taking n / C rows for the
// x transforms; shared memory: the owned columns (n x KC complex), the
// twiddle table (n complex) and one padded n/2-point scratch line per warp. Two
// CTAs per SM when that fits (16 columns at n = 512: clusters of 16 CTAs).
template <int N, int KC_> struct PlaneT {
    static constexpr int M = N / 2;       // complex points of the x transform
    static constexpr int KC = KC_;        // kx columns per CTA
    static constexpr int C = M / KC;      // CTAs per plane
    static constexpr int RY = N / C;      // x rows per CTA
    static constexpr int THREADS = 512;
    static constexpr int WARPS = THREADS / 32;
    static constexpr int EPL = M / 32;    // complex values per lane in a row transform
    static constexpr int SL = M + M / 16;  // scratch line (padded, see spad)
    static constexpr size_t SMEM = ((size_t)N * KC + N + (size_t)WARPS * SL) * sizeof(float2);
    static constexpr int MINB = SMEM <= 110 * 1024 ? 2 : 1;  // resident CTAs per SM
    static constexpr bool OK = (N == 256 || N == 512) && C <= 16 && RY % WARPS == 0 && SMEM <= 200 * 1024;
};

// Cluster barrier without memory ordering: every CTA of the cluster has
// arrived (at the start: all of them run, so their shared memory exists; at
// the end: none still reads another's), nothing published.
__device__ __forceinline__ void cluster_arrive_wait_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}

// Scratch-line index of point i: one pad slot per 16 points, so that the
// first stage's stride-8 writes of a half warp fall in distinct banks.
__device__ __forceinline__ int spad(int i) { return i + (i >> 4); }

// One Stockham stage (radix RAD, sub-length Ns) of the n/2-point transform of
// one row by one warp in its scratch line s: butterfly j reads s[j + r M/RAD]
// and writes s[(j / Ns) Ns RAD + j % Ns + r Ns]. tw: exp(-2 pi i k / N),
// so the stage's twiddle step is N / (Ns RAD).
template <int N, int RAD, bool INV>
__device__ inline void wstage(float2 *s, int Ns, const float2 *tw) {
    constexpr int M = N / 2, B = M / RAD, Q = B / 32;
    static_assert(Q >= 1 && Q * 32 == B, "every lane takes whole butterflies");
    const int lane = (int)threadIdx.x & 31;
    float2 v[Q][RAD];
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < RAD; ++r) v[q][r] = s[spad(lane + 32 * q + r * B)];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = lane + 32 * q, k = j % Ns;
        float2 w1 = tw[k * (N / (Ns * RAD))];
        if (INV) w1.y = -w1.y;
        float2 wr = w1;
#pragma unroll
        for (int r = 1; r < RAD; ++r) {
            v[q][r] = cmul(v[q][r], wr);
            wr = cmul(wr, w1);
        }
        dft_small<RAD, INV>(v[q]);
        const int base = (j / Ns) * Ns * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) s[spad(base + r * Ns)] = v[q][r];
    }
    __syncwarp();
}

// n/2-point complex FFT of one row by one warp, natural order in and out:
// lane l holds v[i] = x[l + 32 i] (the inputs of the first stage, radix
// EPL, whose twiddles are all 1); the result is left in the scratch line s.
// Remaining 32 points: radix 8 then 4 (n = 512) or 4, 4, 2 (n = 256).
template <int N, bool INV>
__device__ inline void warp_fft(float2 (&v)[N / 64], float2 *s, const float2 *tw) {
    constexpr int EPL = N / 64;
    const int lane = (int)threadIdx.x & 31;
    dft_small<EPL, INV>(v);
#pragma unroll
    for (int r = 0; r < EPL; ++r) s[spad(lane * EPL + r)] = v[r];
    __syncwarp();
    if constexpr (EPL == 8) {
        wstage<N, 8, INV>(s, 8, tw);
        wstage<N, 4, INV>(s, 64, tw);
    } else {
        wstage<N, 4, INV>(s, 4, tw);
        wstage<N, 4, INV>(s, 16, tw);
        wstage<N, 2, INV>(s, 64, tw);
    }
}

// One Stockham stage over the KC lines (columns) held as Y[e * KC + line]:
// butterfly b = threadIdx + 512 q takes line b % KC and index j = b / KC.
template <int N, int KC, int RAD, bool INV>
__device__ inline void ystage(float2 *Y, int Ns, const float2 *tw) {
    constexpr int TH = 512;
    constexpr int B = KC * N / RAD, Q = B / TH;
    static_assert(Q >= 1 && Q * TH == B, "every thread takes whole butterflies");
    const int l = (int)threadIdx.x % KC, j0 = (int)threadIdx.x / KC;
    constexpr int JS = TH / KC;  // j stride between a thread's butterflies
    float2 v[Q][RAD];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = j0 + q * JS;
#pragma unroll
        for (int r = 0; r < RAD; ++r) v[q][r] = Y[(j + r * (N / RAD)) * KC + l];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = j0 + q * JS, k = j % Ns;
        if (Ns > 1) {
            float2 w1 = tw[k * (N / (Ns * RAD))];
            if (INV) w1.y = -w1.y;
            float2 wr = w1;
#pragma unroll
            for (int r = 1; r < RAD; ++r) {
                v[q][r] = cmul(v[q][r], wr);
                wr = cmul(wr, w1);
            }
        }
        dft_small<RAD, INV>(v[q]);
        const int base = (j / Ns) * Ns * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) Y[(base + r * Ns) * KC + l] = v[q][r];
    }
    __syncthreads();
}

// n-point FFT along y of the CTA's KC columns, in place (512: 8 8 8; 256: 8 8 4).
template <int N, int KC, bool INV> __device__ inline void y_fft(float2 *Y, const float2 *tw) {
    ystage<N, KC, 8, INV>(Y, 1, tw);
    ystage<N, KC, 8, INV>(Y, 8, tw);
    if constexpr (N == 512) ystage<N, KC, 8, INV>(Y, 64, tw);
    else ystage<N, KC, 4, INV>(Y, 64, tw);
}

// Grid (C, n, members), clusters of C CTAs along x: cluster (z, member)
// transforms plane z. acc: the integer deposit (2^-23 units), kscale = 2^-23 x
// particle mass; spec: the half spectra (z, ky, kx) of every plane; clear:
// zero the accumulator behind the reads (instead of a memset after).
// unit >= 0: the particle mass is 2^(23 - unit), so a kscale - 1 is exactly
// (a - 2^unit) kscale and its rounding to float is that of the integer
// a - 2^unit scaled by the power of two kscale: one 64-bit integer
// subtraction and one conversion instead of two FP64 conversions (the same
// bits as k_acc_mesh); unit < 0 takes the FP64 formula.
template <int N, int KC>
__global__ void __launch_bounds__(512, PlaneT<N, KC>::MINB)
    k_plane_fwd(unsigned long long *__restrict__ acc, float2 *__restrict__ spec, Mesh m, double kscale,
                const float2 *__restrict__ twid, int clear, int unit) {
    typedef PlaneT<N, KC> P;
    constexpr int M = P::M, EPL = P::EPL;
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) float2 psh[];
    float2 *Y = psh, *tw = psh + N * KC;
    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    float2 *s = tw + N + warp * P::SL;
    for (int i = threadIdx.x; i < N; i += P::THREADS) tw[i] = twid[i];
    const int r = (int)cl.block_rank(), z = (int)blockIdx.y;
    const size_t mc = (size_t)blockIdx.z << m.cshift;
    // every CTA of the cluster runs (and the table is loaded) before any
    // row lands in another CTA's columns
    __syncthreads();
    cluster_arrive_wait_relaxed();
    // complex point l + 32 j of a row = its real points 2(l + 32 j), +1; with
    // the register budget of one CTA per SM, the next row's loads are issued
    // before this row's transform
    constexpr bool PREFETCH = P::MINB == 1;
    auto row_of = [&](int i) {
        return reinterpret_cast<ulonglong2 *>(acc + mc + ((size_t)z * N + P::RY * r + i) * N);
    };
    ulonglong2 a[EPL];
    float2 *dst[PREFETCH ? EPL : 1];  // the owners' columns of this lane's kx (same for every row)
    if constexpr (PREFETCH) {
#pragma unroll
        for (int j = 0; j < EPL; ++j) {
            a[j] = __ldcs(row_of(warp) + lane + 32 * j);
            dst[j] = cl.map_shared_rank(Y, (lane + 32 * j) / KC);
        }
    }
    for (int i = warp; i < P::RY; i += P::WARPS) {
        const int y = P::RY * r + i;
        ulonglong2 *row = row_of(i);
        if constexpr (!PREFETCH) {
#pragma unroll
            for (int j = 0; j < EPL; ++j) a[j] = __ldcs(row + lane + 32 * j);
        }
        float2 v[EPL];
        if (unit >= 0) {
            const long long one = 1ll << unit;
            const float fs = (float)kscale;  // a power of two: exact
#pragma unroll
            for (int j = 0; j < EPL; ++j)
                v[j] = make_float2(__ll2float_rn((long long)a[j].x - one) * fs,
                                   __ll2float_rn((long long)a[j].y - one) * fs);
        } else {
#pragma unroll
            for (int j = 0; j < EPL; ++j)
                v[j] = make_float2((float)((double)a[j].x * kscale - 1.0), (float)((double)a[j].y * kscale - 1.0));
        }
        if constexpr (PREFETCH) {
            if (i + P::WARPS < P::RY) {
#pragma unroll
                for (int j = 0; j < EPL; ++j) a[j] = __ldcs(row_of(i + P::WARPS) + lane + 32 * j);
            }
        }
        warp_fft<N, false>(v, s, tw);
        // split: X[k] = (Z[k] + conj Z[M-k]) / 2 - i W^k (Z[k] - conj Z[M-k]) / 2;
        // kx = k goes to column k % KC of CTA k / KC
#pragma unroll
        for (int j = 0; j < EPL; ++j) {
            const int k = lane + 32 * j;
            const float2 za = s[spad(k)], zb = s[spad((M - k) & (M - 1))];
            float2 X;
            if (k == 0) {
                X = make_float2(za.x + za.y, za.x - za.y);  // DC + i Nyquist, both real
            } else {
                const float2 e = make_float2(0.5f * (za.x + zb.x), 0.5f * (za.y - zb.y));  // (Z + conj Zc) / 2
                const float2 o = make_float2(0.5f * (za.y + zb.y), -0.5f * (za.x - zb.x));  // (Z - conj Zc) / 2i
                const float2 t = cmul(tw[k], o);
                X = make_float2(e.x + t.x, e.y + t.y);
            }
            if constexpr (PREFETCH) dst[j][y * KC + k % KC] = X;
            else cl.map_shared_rank(Y, k / KC)[y * KC + k % KC] = X;
        }
        if (clear) {  // the accumulator is read once: leave the row cleared for the next deposit
#pragma unroll
            for (int j = 0; j < EPL; ++j) __stcs(row + lane + 32 * j, make_ulonglong2(0ull, 0ull));
        }
        __syncwarp();  // the scratch line is read before the next row overwrites it
    }
    cl.sync();  // every row's columns have arrived
    y_fft<N, KC, false>(Y, tw);
    float2 *out = spec + (size_t)blockIdx.z * m.mspec + (size_t)z * N * m.nh;
    constexpr int PER = N * KC / P::THREADS;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int e = (int)threadIdx.x + q * P::THREADS, ky = e / KC, c = e % KC;
        const float2 v = Y[e];
        if (r == 0 && c == 0) {  // C[ky] = F0[ky] + i FM[ky] of the two real columns
            const float2 w = Y[((N - ky) & (N - 1)) * KC];
            out[(size_t)ky * m.nh] = make_float2(0.5f * (v.x + w.x), 0.5f * (v.y - w.y));
            out[(size_t)ky * m.nh + M] = make_float2(0.5f * (v.y + w.y), -0.5f * (v.x - w.x));
        } else {
            out[(size_t)ky * m.nh + KC * r + c] = v;
        }
    }
}

// Inverse of k_plane_fwd's transforms (unnormalised, as cuFFT's C2R): half
// spectra (z, ky, kx) -> phi. Same grid and clusters.
template <int N, int KC>
__global__ void __launch_bounds__(512, PlaneT<N, KC>::MINB)
    k_plane_inv(const float2 *__restrict__ spec, float *__restrict__ phi, Mesh m, const float2 *__restrict__ twid) {
    typedef PlaneT<N, KC> P;
    constexpr int M = P::M, EPL = P::EPL;
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ __align__(16) float2 psh[];
    float2 *Y = psh, *tw = psh + N * KC;
    const int warp = (int)threadIdx.x >> 5, lane = (int)threadIdx.x & 31;
    float2 *s = tw + N + warp * P::SL;
    for (int i = threadIdx.x; i < N; i += P::THREADS) tw[i] = twid[i];
    const int r = (int)cl.block_rank(), z = (int)blockIdx.y;
    const float2 *in = spec + (size_t)blockIdx.z * m.mspec + (size_t)z * N * m.nh;
    constexpr int PER = N * KC / P::THREADS, BATCH = (P::MINB == 1 || PER < 8) ? PER : 8;
#pragma unroll
    for (int q0 = 0; q0 < PER; q0 += BATCH) {
        float2 v0[BATCH];  // a batch of the column loads in flight at once
#pragma unroll
        for (int q = 0; q < BATCH; ++q) {
            const int e = (int)threadIdx.x + (q0 + q) * P::THREADS, ky = e / KC, c = e % KC;
            if (r == 0 && c == 0) {  // DC + i Nyquist
                const float2 d = in[(size_t)ky * m.nh], h = in[(size_t)ky * m.nh + M];
                v0[q] = make_float2(d.x - h.y, d.y + h.x);
            } else {
                v0[q] = in[(size_t)ky * m.nh + KC * r + c];
            }
        }
#pragma unroll
        for (int q = 0; q < BATCH; ++q) Y[(int)threadIdx.x + (q0 + q) * P::THREADS] = v0[q];
    }
    __syncthreads();
    y_fft<N, KC, true>(Y, tw);
    cl.sync();  // every CTA's columns are transformed
    const size_t mc = (size_t)blockIdx.z << m.cshift;
    // the row's X[k], k = l + 32 j, from column k % KC of CTA k / KC (X[0]
    // and X[M] are the real and imaginary parts of the packed column); the
    // next row's values are fetched while this row is transformed
    auto fetch = [&](int y, float2 (&x)[EPL]) {
#pragma unroll
        for (int j = 0; j < EPL; ++j) {
            const int k = lane + 32 * j;
            x[j] = cl.map_shared_rank(Y, k / KC)[y * KC + k % KC];
        }
    };
    float2 x[EPL];
    fetch(P::RY * r + warp, x);
    for (int i = warp; i < P::RY; i += P::WARPS) {
        const int y = P::RY * r + i;
#pragma unroll
        for (int j = 0; j < EPL; ++j) s[spad(lane + 32 * j)] = x[j];
        __syncwarp();
        if (i + P::WARPS < P::RY) fetch(y + P::WARPS, x);
        // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k])
        float2 v[EPL];
#pragma unroll
        for (int j = 0; j < EPL; ++j) {
            const int k = lane + 32 * j;
            if (k == 0) {
                const float2 p = s[spad(0)];
                v[j] = make_float2(p.x + p.y, p.x - p.y);
            } else {
                const float2 a = s[spad(k)], b = s[spad(M - k)];
                const float2 e = make_float2(a.x + b.x, a.y - b.y);  // X + conj Xc
                const float2 d = make_float2(a.x - b.x, a.y + b.y);  // X - conj Xc
                const float2 w = make_float2(tw[k].x, -tw[k].y);    // W^-k
                const float2 t = cmul(w, d);
                v[j] = make_float2(e.x - t.y, e.y + t.x);  // e + i t
            }
        }
        __syncwarp();  // X read before the transform overwrites the line
        warp_fft<N, true>(v, s, tw);
        float2 *row = reinterpret_cast<float2 *>(phi + mc + ((size_t)z * N + y) * N);
#pragma unroll
        for (int j = 0; j < EPL; ++j) row[lane + 32 * j] = s[spad(lane + 32 * j)];  // x[2m], x[2m + 1]
        __syncwarp();
    }
    cluster_arrive_wait_relaxed();  // no CTA leaves while another still reads its columns
}

}  // namespace conan
