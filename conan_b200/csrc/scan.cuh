// scan.cuh -- exclusive prefix sum of a uint32 array in three launches
// (block partial sums, a one-block scan of those, block-local scans), used
// for the cell offsets of the counting sorts (deposit, friends-of-friends)
// and the group numbering of friends-of-friends.
#pragma once

#include "common.cuh"

namespace conan {

constexpr unsigned FULL = 0xffffffffu;

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

}  // namespace conan
