// radix.cuh -- stable least-significant-digit radix sort of (uint64 key,
// uint32 value) pairs on the GPU, 8-bit digits, three launches per digit:
//   hist     one CTA per tile of 4096 pairs counts the tile's digits in
//            shared memory; counts stored digit-major (digit x tile);
//   scan     exclusive prefix of the digit-major counts = the first output
//            slot of every (digit, tile);
//   scatter  each warp ranks its 512 pairs per digit in order
//            (__match_any_sync + popc, running per-warp digit counts), the
//            CTA orders the tile by digit in shared memory and writes every
//            digit's run contiguously to its slot.
// Equal digits keep the input order (tile, warp, round, lane), so the passes
// compose into a sort by the whole key that keeps the input order of equal
// keys.
#pragma once

#include "scan.cuh"

namespace conan {

constexpr int RS_T = 256, RS_ITEMS = 16, RS_TILE = RS_T * RS_ITEMS, RS_WARPS = RS_T / 32;
constexpr size_t RS_SMEM = (size_t)RS_TILE * (sizeof(uint64_t) + sizeof(uint32_t));

static __global__ void __launch_bounds__(RS_T) k_rs_hist(const uint64_t *__restrict__ keys, size_t n, int shift,
                                                         uint32_t *__restrict__ bh, unsigned nblk) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * RS_TILE;
#pragma unroll 4
    for (int j = 0; j < RS_ITEMS; ++j) {
        const size_t idx = base + (size_t)j * RS_T + threadIdx.x;
        if (idx < n) atomicAdd(&h[(unsigned)(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    bh[(size_t)threadIdx.x * nblk + blockIdx.x] = h[threadIdx.x];
}

static __global__ void __launch_bounds__(RS_T) k_rs_scatter(const uint64_t *__restrict__ kin,
                                                            const uint32_t *__restrict__ vin, size_t n, int shift,
                                                            const uint32_t *__restrict__ boff, unsigned nblk,
                                                            uint64_t *__restrict__ kout,
                                                            uint32_t *__restrict__ vout) {
    extern __shared__ __align__(16) unsigned char rs_smem[];
    uint64_t *sk = reinterpret_cast<uint64_t *>(rs_smem);
    uint32_t *sv = reinterpret_cast<uint32_t *>(sk + RS_TILE);
    __shared__ uint32_t wh[RS_WARPS][256];  // per-warp digit counts, then per-warp digit bases
    __shared__ uint32_t dstart[256], gbase[256], wsum[RS_WARPS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < RS_WARPS * 256; d += RS_T) (&wh[0][0])[d] = 0;
    __syncthreads();
    const size_t base = (size_t)blockIdx.x * RS_TILE + (size_t)w * (RS_ITEMS * 32);
    const unsigned lt = (1u << lane) - 1u;
    uint64_t k[RS_ITEMS];
    uint32_t v[RS_ITEMS], rk[RS_ITEMS];
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        const size_t idx = base + (size_t)r * 32 + lane;
        const bool ok = idx < n;
        k[r] = ok ? kin[idx] : 0ull;
        v[r] = ok ? vin[idx] : 0u;
        const unsigned d = ok ? ((unsigned)(k[r] >> shift) & 255u) : 256u;
        const unsigned m = __match_any_sync(FULL, d);
        const int leader = __ffs(m) - 1;
        unsigned before = 0;
        if (lane == leader && ok) {
            before = wh[w][d];
            wh[w][d] = before + __popc(m);
        }
        before = __shfl_sync(FULL, before, leader);
        rk[r] = before + __popc(m & lt);
        __syncwarp();
    }
    __syncthreads();
    {
        // thread d: the warps' bases for digit d, the tile's total of d, and
        // the exclusive scan of the totals over the digits
        const int d = threadIdx.x;
        unsigned run = 0;
        for (int ww = 0; ww < RS_WARPS; ++ww) {
            const unsigned c = wh[ww][d];
            wh[ww][d] = run;
            run += c;
        }
        unsigned inc = run;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned u = __shfl_up_sync(FULL, inc, o);
            if (lane >= o) inc += u;
        }
        if (lane == 31) wsum[w] = inc;
        __syncthreads();
        unsigned pre = 0;
        for (int ww = 0; ww < w; ++ww) pre += wsum[ww];
        dstart[d] = pre + inc - run;
        gbase[d] = boff[(size_t)d * nblk + blockIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_ITEMS; ++r) {
        if (base + (size_t)r * 32 + lane < n) {
            const unsigned d = (unsigned)(k[r] >> shift) & 255u;
            const unsigned pos = dstart[d] + wh[w][d] + rk[r];
            sk[pos] = k[r];
            sv[pos] = v[r];
        }
    }
    __syncthreads();
    const size_t tile0 = (size_t)blockIdx.x * RS_TILE;
    const unsigned cnt = (unsigned)((n - tile0) < (size_t)RS_TILE ? (n - tile0) : (size_t)RS_TILE);
    for (unsigned p = threadIdx.x; p < cnt; p += RS_T) {
        const uint64_t key = sk[p];
        const unsigned d = (unsigned)(key >> shift) & 255u;
        const size_t o = (size_t)gbase[d] + (p - dstart[d]);
        kout[o] = key;
        vout[o] = sv[p];
    }
}

// Scratch of radix_sort_pairs for n pairs: digit counts and offsets.
inline size_t radix_tiles(size_t n) { return (n + RS_TILE - 1) / RS_TILE; }

// Sorts n pairs by key bits [0, bits): (k[0], v[0]) in, result in
// (k[w], v[w]) with w the returned index (0 or 1); the other pair of arrays
// is overwritten. bh: 256 * tiles words, boff: 256 * tiles + 1 words, bsum:
// the scan's block sums (one word per SCAN_CHUNK of 256 * tiles).
inline int radix_sort_pairs(uint64_t *k[2], uint32_t *v[2], size_t n, int bits, uint32_t *bh, uint32_t *boff,
                            uint32_t *bsum, cudaStream_t s) {
    const size_t tiles = radix_tiles(n), m = 256 * tiles, nb = (m + SCAN_CHUNK - 1) / SCAN_CHUNK;
    int cur = 0;
    for (int shift = 0; shift < bits; shift += 8) {
        k_rs_hist<<<(unsigned)tiles, RS_T, 0, s>>>(k[cur], n, shift, bh, (unsigned)tiles);
        k_scan_partial<<<(unsigned)nb, SCAN_T, 0, s>>>(bh, m, bsum);
        k_scan_blocks<<<1, 1024, 0, s>>>(bsum, (int)nb);
        k_scan_final<<<(unsigned)nb, SCAN_T, 0, s>>>(bh, m, bsum, boff);
        k_rs_scatter<<<(unsigned)tiles, RS_T, RS_SMEM, s>>>(k[cur], v[cur], n, shift, boff, (unsigned)tiles,
                                                            k[cur ^ 1], v[cur ^ 1]);
        cur ^= 1;
    }
    return cur;
}

}  // namespace conan
