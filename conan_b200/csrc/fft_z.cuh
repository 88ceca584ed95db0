// fft_z.cuh -- the z direction of the Poisson solve's 3D transform, done in
// shared memory with the Green's function multiply in between.
//
// With cuFFT's 2D R2C over every z plane of the density, the half spectrum of
// one member is (z, ky, kx) with kx fastest: z still in real space. One CTA
// takes TX consecutive kx columns of one ky row, i.e. TX complex lines of n
// values along z (stride n * nh), and runs
//   forward complex FFT along z (natural order out)
//   spec *= gs / |k|^2, DC = 0 (the multiply of k_green: same formula)
//   inverse complex FFT along z (unnormalised)
// in shared memory, so the spectrum crosses HBM once between the forward and
// the inverse 2D transforms instead of three times (3D transforms' z passes
// and the multiply). The 2D C2R per plane then gives phi.
//
// The FFT is the Stockham self-sorting formulation (Govindaraju et al.,
// "High performance discrete Fourier transforms on graphics processors",
// SC 2008): stage with sub-length Ns and radix R reads x[j + r N/R], applies
// the twiddles exp(-+2 pi i (j mod Ns) r / (Ns R)), a radix-R DFT in
// registers, and writes x[(j / Ns) Ns R + (j mod Ns) + r Ns]. Radix 8
// stages, then one radix-2 or radix-4 stage for n = 8^a * {1, 2, 4}. Each
// stage reads all its inputs, synchronises, and writes in place. Twiddles
// come from a table of exp(-2 pi i k / n) computed in double on the host.
#pragma once

#include "common.cuh"

namespace conan {

// Lines per CTA and threads per CTA for an n-point z transform: n / 8
// threads per line (n / 16 from 256 points up). (At n = 1024, 4 lines per CTA instead of 8 measured
// slower: 31.0 against 30.0 ms per step of the 1024^3-mesh run.)
// TX = 0 takes the default width; the autotuner also tries half and twice
// the default (ZTile<N, TX>::OK says whether a width fits one CTA).
// Threads per line at 1024 points: 128 (one radix-8 butterfly per thread
// and stage, one 1024-thread CTA per SM) or 64 (two butterflies, two
// 512-thread CTAs per SM: 4.27 against 4.85 ms per pass on the 1024^3
// mesh); a compile-time tunable.
#ifndef ZPASS_LT1024
#define ZPASS_LT1024 64
#endif
// The same at 512 points: 64, 32 or 16 threads per line (0.385, 0.371 and
// 0.384 ms per pass on the 512^3 mesh), and at 256 points 32 or 16 (0.050
// and 0.047 ms on the 256^3 mesh).
#ifndef ZPASS_LT512
#define ZPASS_LT512 32
#endif
#ifndef ZPASS_LT256
#define ZPASS_LT256 16
#endif
template <int N, int TX_ = 0> struct ZTile {
    static constexpr int TX = TX_ ? TX_ : (N >= 256 ? 8 : 2048 / N);
    static constexpr int LT = N == 1024 ? ZPASS_LT1024 : N == 512 ? ZPASS_LT512 : N == 256 ? ZPASS_LT256 : N / 8;  // threads per line
    static constexpr int THREADS = TX * LT;
    static constexpr size_t SMEM = (size_t)TX * N * sizeof(float2) + (size_t)N * sizeof(float2);
    static constexpr bool OK = THREADS <= 1024 && SMEM <= 200 * 1024;
};

__device__ inline float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ inline float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ inline float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// times -i (forward) or +i (inverse)
template <bool INV> __device__ inline float2 cmul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// In-register DFT of RAD = 2, 4 or 8 values, natural order in and out
// (radix-2 decimation in frequency, outputs unscrambled by bit reversal).
template <int RAD, bool INV> __device__ inline void dft_small(float2 *v) {
    if constexpr (RAD == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (RAD == 4) {
        const float2 a0 = cadd(v[0], v[2]), a2 = csub(v[0], v[2]);
        const float2 a1 = cadd(v[1], v[3]), a3 = cmul_mi<INV>(csub(v[1], v[3]));
        v[0] = cadd(a0, a1);
        v[2] = csub(a0, a1);
        v[1] = cadd(a2, a3);
        v[3] = csub(a2, a3);
    } else {
        const float h = 0.70710678118654752440f;  // 1 / sqrt(2)
        float2 a[8];
        a[0] = cadd(v[0], v[4]);
        a[1] = cadd(v[1], v[5]);
        a[2] = cadd(v[2], v[6]);
        a[3] = cadd(v[3], v[7]);
        a[4] = csub(v[0], v[4]);
        const float2 d1 = csub(v[1], v[5]), d3 = csub(v[3], v[7]);
        // d1 * W8, d2 * W8^2, d3 * W8^3 with W8 = exp(-+ i pi / 4)
        a[5] = INV ? make_float2((d1.x - d1.y) * h, (d1.x + d1.y) * h) : make_float2((d1.x + d1.y) * h, (d1.y - d1.x) * h);
        a[6] = cmul_mi<INV>(csub(v[2], v[6]));
        a[7] = INV ? make_float2(-(d3.x + d3.y) * h, (d3.x - d3.y) * h) : make_float2((d3.y - d3.x) * h, -(d3.x + d3.y) * h);
        float2 b[8];
        b[0] = cadd(a[0], a[2]);
        b[1] = cadd(a[1], a[3]);
        b[2] = csub(a[0], a[2]);
        b[3] = cmul_mi<INV>(csub(a[1], a[3]));
        b[4] = cadd(a[4], a[6]);
        b[5] = cadd(a[5], a[7]);
        b[6] = csub(a[4], a[6]);
        b[7] = cmul_mi<INV>(csub(a[5], a[7]));
        v[0] = cadd(b[0], b[1]);
        v[4] = csub(b[0], b[1]);
        v[2] = cadd(b[2], b[3]);
        v[6] = csub(b[2], b[3]);
        v[1] = cadd(b[4], b[5]);
        v[5] = csub(b[4], b[5]);
        v[3] = cadd(b[6], b[7]);
        v[7] = csub(b[6], b[7]);
    }
}

// Where a stage reads from and writes to: shared memory (value index e of
// line l at buf[e * TX + l]) or the spectrum in global memory (value e of line
// l at g[e * zs + l], lines at or beyond `valid` neither read nor written).
struct ZIO {
    float2 *buf;
    float2 *g;
    size_t zs;
    int valid;
};

// Green's function of the value at z index e of line l: the multiply of
// k_green with kz = wave(e).
struct ZGreen {
    long long kyy;  // ky^2 of the row
    int kx0;        // kx of line 0
    int n;
    float gs;
    __device__ inline float operator()(int e, int l) const {
        const int kz = e > n / 2 ? e - n : e;
        const int k2 = (kx0 + l) * (kx0 + l) + (int)kyy + kz * kz;  // <= 3 (n/2)^2: fits 32 bits
        return k2 > 0 ? __fdividef(gs, (float)k2) : 0.0f;
    }
};

// One Stockham stage of radix RAD with sub-length Ns. IN_G / OUT_G: read from
// / write to global memory instead of shared memory; GREEN: multiply the
// inputs by the Green's function first.
template <int N, int TXW, int RAD, bool INV, bool IN_G, bool OUT_G, bool GREEN>
__device__ inline void zstage(const ZIO &io, int Ns, const float2 *tw, const ZGreen &gf) {
    constexpr int TX = ZTile<N, TXW>::TX, LT = ZTile<N, TXW>::LT;
    constexpr int NB = N / RAD;  // butterflies per line
    constexpr int Q = NB / LT;   // butterflies per thread
    const int l = (int)threadIdx.x % TX, j0 = (int)threadIdx.x / TX;
    float2 v[Q][RAD];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = j0 + q * LT;
#pragma unroll
        for (int r = 0; r < RAD; ++r) {
            const int e = j + r * NB;
            float2 x;
            if constexpr (IN_G) x = l < io.valid ? io.g[(size_t)e * io.zs + l] : make_float2(0.f, 0.f);
            else x = io.buf[e * TX + l];
            if constexpr (GREEN) {
                const float g = gf(e, l);
                x.x *= g;
                x.y *= g;
            }
            v[q][r] = x;
        }
    }
    if constexpr (!IN_G) __syncthreads();  // every input read before any output lands in place
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = j0 + q * LT, k = j % Ns;
        const int step = N / (Ns * RAD);
        if (Ns > 1) {  // the first stage's twiddles are all exactly 1
            // w^r by recurrence from one table entry (one shared-memory load
            // instead of RAD - 1: 0.45 -> 0.42 ms at 512^3)
            float2 w1 = tw[(k * step) & (N - 1)];
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
        for (int r = 0; r < RAD; ++r) {
            const int e = base + r * Ns;
            if constexpr (OUT_G) {
                if (l < io.valid) io.g[(size_t)e * io.zs + l] = v[q][r];
            } else {
                io.buf[e * TX + l] = v[q][r];
            }
        }
    }
    if constexpr (!OUT_G) __syncthreads();
}

// The forward transform's last stage (radix 8, sub-length N/8), the Green
// multiply and the inverse transform's first stage (radix 8, sub-length 1)
// in registers: thread j's eight outputs x[j + r N/8] of the one are the
// eight inputs of the other, so the two stages share one shared-memory
// round trip.
template <int N, int TXW>
__device__ inline void zstage_mid(const ZIO &io, const float2 *tw, const ZGreen &gf) {
    constexpr int TX = ZTile<N, TXW>::TX, LT = ZTile<N, TXW>::LT, NB = N / 8, Q = NB / LT;
    static_assert(Q * LT == NB, "whole radix-8 butterflies per thread");
    const int l = (int)threadIdx.x % TX, j0 = (int)threadIdx.x / TX;
    float2 v[Q][8];
#pragma unroll
    for (int q = 0; q < Q; ++q)
#pragma unroll
        for (int r = 0; r < 8; ++r) v[q][r] = io.buf[(j0 + q * LT + r * NB) * TX + l];
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = j0 + q * LT;
        // forward: twiddles exp(-2 pi i j r / N), then the radix-8 DFT
        const float2 w1 = tw[j];
        float2 wr = w1;
#pragma unroll
        for (int r = 1; r < 8; ++r) {
            v[q][r] = cmul(v[q][r], wr);
            wr = cmul(wr, w1);
        }
        dft_small<8, false>(v[q]);
        // natural-order index j + r N/8: the Green's function, then the
        // inverse first stage (all twiddles 1) writing x[8 j + r]
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const float g = gf(j + r * NB, l);
            v[q][r].x *= g;
            v[q][r].y *= g;
        }
        dft_small<8, true>(v[q]);
#pragma unroll
        for (int r = 0; r < 8; ++r) io.buf[(8 * j + r) * TX + l] = v[q][r];
    }
    __syncthreads();
}

// Radix of stage s of an n-point transform: 8 while 8 divides the rest.
template <int N> struct ZRadix {
    static constexpr int S8 = N >= 512 ? 3 : 2;  // radix-8 stages (64..1024 points)
    static constexpr int REST = N / (S8 == 3 ? 512 : 64);  // 1, 2 or 4
};

// Forward z FFT, Green multiply, inverse z FFT for TX columns of one row.
// Grid: (ceil(nh / TX), n rows ky, members). spec: the members' half spectra
// after the 2D transforms of every z plane.
#ifndef ZPASS_MIN_BLOCKS
#define ZPASS_MIN_BLOCKS 3  // resident CTAs per SM the register budget must allow (measured: 0.45 against 0.51 ms with 1 at 512^3)
#endif

template <int N, int TXW = 0>
__global__ void __launch_bounds__(ZTile<N, TXW>::THREADS,
                                  ZTile<N, TXW>::THREADS >= 1024 ? 1 : ZTile<N, TXW>::LT < N / 8 ? 2 : ZPASS_MIN_BLOCKS)
    k_zpass_green(float2 *__restrict__ spec, Mesh m, float gs,
                                                                   const float2 *__restrict__ twid) {
    extern __shared__ __align__(16) float2 zsh[];
    constexpr int TX = ZTile<N, TXW>::TX;
    float2 *tw = zsh + TX * N;
    for (int i = threadIdx.x; i < N; i += ZTile<N, TXW>::THREADS) tw[i] = twid[i];
    __syncthreads();
    const int kx0 = (int)blockIdx.x * TX, ky = (int)blockIdx.y;
    const size_t zs = (size_t)m.n * m.nh;
    ZIO io{zsh, spec + (size_t)blockIdx.z * m.mspec + (size_t)ky * m.nh + kx0, zs, m.nh - kx0};
    const int wy = wave_index(ky, m.n);
    const ZGreen gf{(long long)wy * wy, kx0, m.n, gs};
    constexpr int S8 = ZRadix<N>::S8, REST = ZRadix<N>::REST;
    // forward: the radix-2/4 stage first (from global memory) when n is not
    // a power of 8, then the radix-8 stages, the last of them fused with the
    // Green multiply and the inverse's first stage (zstage_mid); the inverse
    // goes on with radix 8 and ends with the radix-2/4 stage (to global)
    int Ns = 1;
    if constexpr (REST > 1) {
        zstage<N, TXW, REST, false, true, false, false>(io, Ns, tw, gf);
        Ns *= REST;
        zstage<N, TXW, 8, false, false, false, false>(io, Ns, tw, gf);
        Ns *= 8;
    } else {
        zstage<N, TXW, 8, false, true, false, false>(io, Ns, tw, gf);
        Ns *= 8;
    }
#pragma unroll
    for (int s = 2; s < S8; ++s, Ns *= 8) zstage<N, TXW, 8, false, false, false, false>(io, Ns, tw, gf);
    zstage_mid<N, TXW>(io, tw, gf);
    Ns = 8;
    if constexpr (REST > 1) {
#pragma unroll
        for (int s = 1; s < S8; ++s, Ns *= 8) zstage<N, TXW, 8, true, false, false, false>(io, Ns, tw, gf);
        zstage<N, TXW, REST, true, false, true, false>(io, Ns, tw, gf);
    } else {
#pragma unroll
        for (int s = 1; s < S8 - 1; ++s, Ns *= 8) zstage<N, TXW, 8, true, false, false, false>(io, Ns, tw, gf);
        zstage<N, TXW, 8, true, false, true, false>(io, Ns, tw, gf);
    }
}

}  // namespace conan
