// Single-pass exclusive prefix sum over uint32 (decoupled look-back), for sm_100a.
//
// Replaces the reference's cub::DeviceScan::ExclusiveSum call (Wrappers.cu:125-136). One pass over
// the data: each tile reads its items once and writes its outputs once (8 bytes per item of HBM
// traffic), so the kernel is bound by HBM bandwidth.
//
// Tiles are claimed in order through an atomic ticket, so every tile a thread block waits on was
// claimed by a block that is already running: the look-back always makes progress. Every wait is
// still bounded (kMaxPolls); on expiry the kernel records a timeout in Diag and continues with the
// value it has, so the host sees an error status instead of a hung GPU.
#pragma once

#include "sdf_device.cuh"

namespace sdfb {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ROUNDS = 4;                                  // uint4 loads per thread
constexpr int SCAN_TILE = SCAN_THREADS * 4 * SCAN_ROUNDS;       // 4096 items per tile
constexpr unsigned long long FLAG_AGG = 1ull << 32;             // tile aggregate published
constexpr unsigned long long FLAG_PFX = 2ull << 32;             // inclusive prefix published
constexpr int kMaxPolls = 1 << 22;

struct ScanState {
    unsigned long long* status;  // one word per tile: flag << 32 | value
    unsigned int* ticket;        // tile ticket counter
};

__device__ __forceinline__ unsigned long long ld_status(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_status(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// exclusive block scan of one value per thread; returns the exclusive prefix, *total = block sum
template <int THREADS>
__device__ __forceinline__ unsigned block_exclusive(unsigned v, unsigned* smem_warp, unsigned* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        unsigned w = (lane < THREADS / 32) ? smem_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < THREADS / 32) smem_warp[lane] = w;  // inclusive warp prefixes
    }
    __syncthreads();
    const unsigned warp_base = warp ? smem_warp[warp - 1] : 0u;
    *total = smem_warp[THREADS / 32 - 1];
    __syncthreads();
    return warp_base + x - v;
}

// Decoupled look-back for the tile `tile` whose aggregate is `agg` (called by all threads; the
// returned exclusive prefix is valid in every thread).
__device__ __forceinline__ unsigned tile_lookback(const ScanState& st, int tile, unsigned agg, unsigned* smem_pfx,
                                                  Diag* diag) {
    if (threadIdx.x == 0) {
        if (tile == 0) {
            st_status(&st.status[0], FLAG_PFX | agg);
            *smem_pfx = 0;
        } else {
            st_status(&st.status[tile], FLAG_AGG | agg);
        }
    }
    if (tile != 0 && threadIdx.x < 32) {
        const int lane = threadIdx.x;
        unsigned excl = 0;
        int base = tile - 1;
        bool done = false;
        bool timed_out = false;
        while (!done) {
            // look at the 32 predecessors [base-31, base]; lane 0 = the nearest
            const int idx = base - lane;
            unsigned long long s = 0;
            int polls = 0;
            if (idx >= 0) {
                s = ld_status(&st.status[idx]);
                while ((s >> 32) == 0 && polls < kMaxPolls) {
                    s = ld_status(&st.status[idx]);
                    ++polls;
                }
                if ((s >> 32) == 0) timed_out = true;
            } else {
                s = FLAG_PFX;  // before tile 0: prefix 0
            }
            const unsigned is_pfx = __ballot_sync(0xffffffffu, (s >> 32) >= 2);
            // sum the aggregates up to and including the nearest published prefix
            const int stop = is_pfx ? __ffs(is_pfx) - 1 : 31;
            unsigned v = (lane <= stop) ? (unsigned)(s & 0xffffffffu) : 0u;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            excl += v;
            if (is_pfx) done = true;
            base -= 32;
            if (__any_sync(0xffffffffu, timed_out)) break;
        }
        if (lane == 0) {
            st_status(&st.status[tile], FLAG_PFX | (unsigned)(excl + agg));
            *smem_pfx = excl;
            if (timed_out && diag) atomicExch(&diag->timeout, 1);
        }
    }
    __syncthreads();
    const unsigned r = *smem_pfx;
    __syncthreads();
    return r;
}

// out[i] = sum(in[0..i)), i < n. n is min(*n_dev, n_host) * n_mult when n_dev != nullptr (a device-side
// count, bounded by the rows the arrays hold), else n_host. If `total` is set, the grand total is written there by the last tile.
__global__ void __launch_bounds__(SCAN_THREADS) k_exclusive_scan(const unsigned* __restrict__ in,
                                                                 unsigned* __restrict__ out, unsigned n_host,
                                                                 const int* __restrict__ n_dev, unsigned n_mult,
                                                                 ScanState st, unsigned* total, Diag* diag) {
    __shared__ unsigned s_warp[SCAN_THREADS / 32];
    __shared__ unsigned s_pfx;
    __shared__ int s_tile;
    // with a device count, n_host bounds it (the rows the caller's arrays hold)
    const unsigned n = n_dev ? (unsigned)min(max(*n_dev, 0), (int)n_host) * n_mult : n_host;
    if (threadIdx.x == 0) s_tile = (int)atomicAdd(st.ticket, 1u);
    __syncthreads();
    const int tile = s_tile;
    const unsigned base = (unsigned)tile * SCAN_TILE;
    if (base >= n && tile != 0) return;
    if (n == 0) {
        if (total && threadIdx.x == 0) *total = 0;
        return;
    }
    // load: round r covers items [base + r*1024, +1024), 4 per thread
    uint4 v[SCAN_ROUNDS];
    unsigned tsum[SCAN_ROUNDS];
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) {
        const unsigned i0 = base + (unsigned)r * (SCAN_THREADS * 4) + threadIdx.x * 4;
        if (i0 + 3 < n && ((reinterpret_cast<uintptr_t>(in) & 15) == 0)) {
            v[r] = __ldcs(reinterpret_cast<const uint4*>(in + i0));
        } else {
            v[r].x = i0 < n ? in[i0] : 0u;
            v[r].y = i0 + 1 < n ? in[i0 + 1] : 0u;
            v[r].z = i0 + 2 < n ? in[i0 + 2] : 0u;
            v[r].w = i0 + 3 < n ? in[i0 + 3] : 0u;
        }
        tsum[r] = v[r].x + v[r].y + v[r].z + v[r].w;
    }
    unsigned pre[SCAN_ROUNDS], rtot[SCAN_ROUNDS];
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) pre[r] = block_exclusive<SCAN_THREADS>(tsum[r], s_warp, &rtot[r]);
    unsigned agg = 0;
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) agg += rtot[r];
    const unsigned tile_pfx = tile_lookback(st, tile, agg, &s_pfx, diag);
    unsigned carry = tile_pfx;
#pragma unroll
    for (int r = 0; r < SCAN_ROUNDS; ++r) {
        const unsigned i0 = base + (unsigned)r * (SCAN_THREADS * 4) + threadIdx.x * 4;
        uint4 o;
        o.x = carry + pre[r];
        o.y = o.x + v[r].x;
        o.z = o.y + v[r].y;
        o.w = o.z + v[r].z;
        if (i0 + 3 < n && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
            __stcs(reinterpret_cast<uint4*>(out + i0), o);
        } else {
            if (i0 < n) out[i0] = o.x;
            if (i0 + 1 < n) out[i0 + 1] = o.y;
            if (i0 + 2 < n) out[i0 + 2] = o.z;
            if (i0 + 3 < n) out[i0 + 3] = o.w;
        }
        carry += rtot[r];
    }
    if (total && threadIdx.x == 0 && base + SCAN_TILE >= n) *total = tile_pfx + agg;
}

inline unsigned scan_tiles(unsigned n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

}  // namespace sdfb
