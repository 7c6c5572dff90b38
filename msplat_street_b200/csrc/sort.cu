// Tile-intersection binning: exclusive scan, key emission, stable LSD radix sort and
// tile ranges.
//
// The reference builds per-tile lists ordered by (depth bits, Gaussian index)
// (bin_and_sort, core/cpu/msplat_cpu.cpp:505-567). Here every (Gaussian, tile) pair
// gets one 64-bit key (tile id << 32) | depth bits, written in Gaussian order at
// offsets from an exclusive scan of tiles-per-Gaussian. A STABLE radix sort over the
// significant bits then yields, within each tile, ascending depth with ties in
// Gaussian order -- exactly the reference's order -- without a per-tile sort or any
// cap on a tile's list. The sort carries the emission index as its value; the map
// kernel turns it into the Gaussian id per sorted slot and the inverse permutation
// that the backward pass uses to reduce per-Gaussian gradients deterministically.
//
// The radix sort is reduce-then-scan per 8-bit digit: a histogram kernel, a device
// scan of the digit-major counts, and a scatter kernel that ranks keys stably inside
// each 2048-key block with warp match/popc. No block waits on another block.
#include <algorithm>

#include "common.cuh"
#include "kernels.h"

namespace msplat {

// ---------------------------------------------------------------------------------
// Exclusive scan (int32 in, TO out), 2048 elements per block, three kernels.

constexpr int SCAN_THREADS = 256, SCAN_ITEMS = 8, SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T *warp_sums, T &block_total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : T(0);
        T wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T t = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += t;
        }
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = wi - w;
        if (lane == 31) warp_sums[32] = wi;
    }
    __syncthreads();
    T r = warp_sums[warp] + inc - v;
    block_total = warp_sums[32];
    __syncthreads();
    return r;
}

template <typename TO>
__global__ void scan_reduce_kernel(const int32_t *in, int n, TO *partials) {
    __shared__ TO ws[33];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    TO s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; j++)
        if (base + j < n) s += (TO)in[base + j];
    TO tot;
    block_exclusive_scan<TO>(s, ws, tot);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

template <typename TO>
__global__ void scan_partials_kernel(TO *partials, int nb, TO *total) {
    __shared__ TO ws[33];
    TO carry = 0;
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        TO v = i < nb ? partials[i] : TO(0);
        TO tot;
        TO ex = block_exclusive_scan<TO>(v, ws, tot);
        if (i < nb) partials[i] = ex + carry;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <typename TO>
__global__ void scan_apply_kernel(const int32_t *in, int n, const TO *partials, TO *out) {
    __shared__ TO ws[33];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_ITEMS;
    TO v[SCAN_ITEMS];
    TO s = 0;
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; j++) {
        v[j] = base + j < n ? (TO)in[base + j] : TO(0);
        s += v[j];
    }
    TO tot;
    TO ex = block_exclusive_scan<TO>(s, ws, tot) + partials[blockIdx.x];
#pragma unroll
    for (int j = 0; j < SCAN_ITEMS; j++) {
        if (base + j < n) out[base + j] = ex;
        ex += v[j];
    }
}

int scan_blocks(int n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

template <typename TO>
void scan_exclusive(const int32_t *in, TO *out, int n, TO *d_total, TO *partials, cudaStream_t st) {
    if (n <= 0) {
        if (d_total) cudaMemsetAsync(d_total, 0, sizeof(TO), st);
        return;
    }
    const int nb = scan_blocks(n);
    scan_reduce_kernel<TO><<<nb, SCAN_THREADS, 0, st>>>(in, n, partials);
    scan_partials_kernel<TO><<<1, 1024, 0, st>>>(partials, nb, d_total);
    scan_apply_kernel<TO><<<nb, SCAN_THREADS, 0, st>>>(in, n, partials, out);
}
template void scan_exclusive<int32_t>(const int32_t *, int32_t *, int, int32_t *, int32_t *, cudaStream_t);
template void scan_exclusive<int64_t>(const int32_t *, int64_t *, int, int64_t *, int64_t *, cudaStream_t);

// ---------------------------------------------------------------------------------
// Key emission: one thread per Gaussian, tiles in row-major order of its rectangle.

__device__ __forceinline__ void rect_of(const Splat &s, float ax, float ay, int tx, int ty, int &x0, int &y0, int &x1,
                                        int &y1) {
    float ccx = s.x / (float)TILE, ccy = s.y / (float)TILE;
    float rrx = ax / (float)TILE, rry = ay / (float)TILE;
    x0 = min(max(0, (int)(ccx - rrx)), tx);
    x1 = min(max(0, (int)(ccx + rrx + 1)), tx);
    y0 = min(max(0, (int)(ccy - rry)), ty);
    y1 = min(max(0, (int)(ccy + rry + 1)), ty);
}

__global__ void emit_keys_kernel(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles,
                                 const int64_t *offsets, int tiles_x, int tiles_y, uint64_t *keys, uint32_t *vals,
                                 int32_t *emit_gid) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || n_tiles[i] <= 0) return;
    const Splat s = splats[i];
    int x0, y0, x1, y1;
    rect_of(s, aabb[2 * i], aabb[2 * i + 1], tiles_x, tiles_y, x0, y0, x1, y1);
    const uint64_t db = (uint64_t)__float_as_uint(s.depth);
    int64_t e = offsets[i];
    for (int y = y0; y < y1; y++)
        for (int x = x0; x < x1; x++, e++) {
            keys[e] = ((uint64_t)(y * tiles_x + x) << 32) | db;
            vals[e] = (uint32_t)e;
            emit_gid[e] = i;
        }
}

void launch_emit_keys(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles, const int64_t *offsets,
                      int tiles_x, int tiles_y, uint64_t *keys, uint32_t *vals, int32_t *emit_gid, cudaStream_t st) {
    if (n <= 0) return;
    emit_keys_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, splats, aabb, n_tiles, offsets, tiles_x, tiles_y, keys, vals,
                                                      emit_gid);
}

// Batched emission: instance g (a Gaussian of one view) keys its tiles with the
// view's first global tile added, so one stable sort orders every view's tiles at
// once and each tile's list is the one the single-view sort gives.
__global__ void emit_keys_batch_kernel(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles,
                                       const int64_t *offsets, const BatchDesc d, uint64_t *keys, uint32_t *vals,
                                       int32_t *emit_gid, int64_t cap) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n || n_tiles[g] <= 0) return;
    const int v = find_view(d.inst_off, d.n_views, g);
    const int tiles_x = d.tiles_x[v], tiles_y = d.tiles_y[v];
    const uint64_t base = (uint64_t)d.tile_off[v];
    const Splat s = splats[g];
    int x0, y0, x1, y1;
    rect_of(s, aabb[2 * g], aabb[2 * g + 1], tiles_x, tiles_y, x0, y0, x1, y1);
    const uint64_t db = (uint64_t)__float_as_uint(s.depth);
    int64_t e = offsets[g];
    for (int y = y0; y < y1; y++)
        for (int x = x0; x < x1 && e < cap; x++, e++) {  // cap: buffer capacity (graph mode)
            keys[e] = ((base + (uint64_t)(y * tiles_x + x)) << 32) | db;
            vals[e] = (uint32_t)e;
            emit_gid[e] = g;
        }
}

void launch_emit_keys_batch(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles,
                            const int64_t *offsets, const BatchDesc &d, uint64_t *keys, uint32_t *vals,
                            int32_t *emit_gid, cudaStream_t st, int64_t cap) {
    if (n <= 0) return;
    emit_keys_batch_kernel<<<(n + 127) / 128, 128, 0, st>>>(n, splats, aabb, n_tiles, offsets, d, keys, vals,
                                                            emit_gid, cap);
}

// ---------------------------------------------------------------------------------
// Stable LSD radix sort of (u64 key, u32 value) by key bits [0, key_bits).

constexpr int RADIX = 256;
constexpr int SORT_THREADS = 256, SORT_WARPS = SORT_THREADS / 32, SORT_ITEMS = 8;
constexpr int SORT_TILE = SORT_THREADS * SORT_ITEMS;  // keys per block
constexpr int WARP_KEYS = SORT_TILE / SORT_WARPS;     // contiguous keys per warp

int radix_blocks(int n) { return (n + SORT_TILE - 1) / SORT_TILE; }

// d_n (may be null): a device-side count that caps n (capacity-bounded launches)
__global__ void radix_hist_kernel(const uint64_t *keys, int n, const int *d_n, int shift, uint32_t mask,
                                  uint32_t *counts, int nb) {
    __shared__ uint32_t h[RADIX];
    if (d_n) n = min(n, *d_n);
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int base = blockIdx.x * SORT_TILE;
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {
        const int k = base + j * SORT_THREADS + threadIdx.x;
        const bool ok = k < n;
        const int d = ok ? (int)((keys[k] >> shift) & mask) : RADIX;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (ok && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x) counts[(size_t)i * nb + blockIdx.x] = h[i];
}

// counts -> exclusive digit-major offsets (uint32 scan over 256 * nb entries)
__global__ void radix_scatter_kernel(const uint64_t *kin, const uint32_t *vin, uint64_t *kout, uint32_t *vout, int n,
                                     const int *d_n, int shift, uint32_t mask, const int32_t *offs, int nb) {
    __shared__ uint32_t wcnt[SORT_WARPS][RADIX];
    __shared__ uint32_t gbase[RADIX];
    if (d_n) n = min(n, *d_n);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < SORT_WARPS * RADIX; i += blockDim.x) (&wcnt[0][0])[i] = 0;
    for (int i = threadIdx.x; i < RADIX; i += blockDim.x) gbase[i] = (uint32_t)offs[(size_t)i * nb + blockIdx.x];
    __syncthreads();
    uint64_t key[SORT_ITEMS];
    uint32_t val[SORT_ITEMS], rank[SORT_ITEMS];
    int dig[SORT_ITEMS];
    const int base = blockIdx.x * SORT_TILE + warp * WARP_KEYS;
    const unsigned lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {
        const int k = base + r * 32 + lane;
        const bool ok = k < n;
        key[r] = ok ? kin[k] : 0ull;
        val[r] = ok ? vin[k] : 0u;
        const int d = ok ? (int)((key[r] >> shift) & mask) : RADIX;
        dig[r] = d;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = ok ? wcnt[warp][d] : 0u;
        rank[r] = before + (uint32_t)__popc(peers & lt);
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] = before + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    for (int d = threadIdx.x; d < RADIX; d += blockDim.x) {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < SORT_WARPS; w++) {
            const uint32_t t = wcnt[w][d];
            wcnt[w][d] = run;
            run += t;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {
        const int k = base + r * 32 + lane;
        if (k < n) {
            const int d = dig[r];
            const uint32_t pos = gbase[d] + wcnt[warp][d] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
}

size_t radix_scratch_bytes(int n) {
    const int nb = radix_blocks(n > 1 ? n : 1);
    const size_t cnt = (size_t)RADIX * nb;
    return cnt * sizeof(int32_t) * 2 + (size_t)scan_blocks((int)cnt) * sizeof(int32_t) + 64;
}

// Sorts (k[0], v[0]) using (k[1], v[1]) as the ping-pong buffers; returns the index
// (0 or 1) of the buffer pair holding the result. With d_n, n is a capacity and the
// count is read on the device (no host round trip; every pass runs).
int radix_sort_pairs(uint64_t *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st,
                     const int *d_n) {
    if ((!d_n && n <= 1) || n <= 0 || key_bits <= 0) return 0;
    const int nb = radix_blocks(n);
    const size_t cnt = (size_t)RADIX * nb;
    int32_t *counts = reinterpret_cast<int32_t *>(scratch);
    int32_t *offs = counts + cnt;
    int32_t *partials = offs + cnt;
    int cur = 0;
    for (int shift = 0; shift < key_bits; shift += 8) {
        const int bits = key_bits - shift < 8 ? key_bits - shift : 8;  // digits above key_bits are ignored
        const uint32_t mask = (1u << bits) - 1u;
        radix_hist_kernel<<<nb, SORT_THREADS, 0, st>>>(k[cur], n, d_n, shift, mask,
                                                       reinterpret_cast<uint32_t *>(counts), nb);
        scan_exclusive<int32_t>(counts, offs, (int)cnt, nullptr, partials, st);
        radix_scatter_kernel<<<nb, SORT_THREADS, 0, st>>>(k[cur], v[cur], k[cur ^ 1], v[cur ^ 1], n, d_n, shift, mask,
                                                          offs, nb);
        cur ^= 1;
    }
    return cur;
}

// ---------------------------------------------------------------------------------
// Tile ranges by binary search (empty tiles get start == end == the running count,
// as the reference's prefix sums give), and the per-slot Gaussian id / inverse map.

__global__ void tile_ranges_kernel(const uint64_t *keys, int n, int T, int32_t *tile_start, int32_t *tile_end,
                                   const int *d_n, const int *d_T) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_n) n = min(n, *d_n);
    if (d_T) T = min(T, *d_T);
    if (t > T) return;
    int lo = 0, hi = n;  // first position whose tile id >= t
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((int)(keys[mid] >> 32) < t) lo = mid + 1;
        else hi = mid;
    }
    if (t < T) tile_start[t] = lo;
    if (t > 0) tile_end[t - 1] = lo;
}

__global__ void isect_map_kernel(const uint32_t *sorted_e, int n, const int32_t *emit_gid, int32_t *isect_gid,
                                 int32_t *inv, const int *d_n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_n) n = min(n, *d_n);
    if (k >= n) return;
    const uint32_t e = sorted_e[k];
    isect_gid[k] = emit_gid[e];
    inv[e] = k;
}

void launch_tile_ranges(const uint64_t *keys, int n, int T, int32_t *tile_start, int32_t *tile_end, cudaStream_t st,
                        const int *d_n, const int *d_T) {
    tile_ranges_kernel<<<(T + 1 + 255) / 256, 256, 0, st>>>(keys, n, T, tile_start, tile_end, d_n, d_T);
}

void launch_isect_map(const uint32_t *sorted_e, int n, const int32_t *emit_gid, int32_t *isect_gid, int32_t *inv,
                      cudaStream_t st, const int *d_n) {
    if (n <= 0) return;
    isect_map_kernel<<<(n + 255) / 256, 256, 0, st>>>(sorted_e, n, emit_gid, isect_gid, inv, d_n);
}

// Device-side intersection count for capacity-bounded (graph-capturable) steps:
// d_n = total when it fits the capacity, else 0 with *overflow set (the step then
// renders nothing and updates nothing; the host grows the buffers and repeats it).
__global__ void clamp_count_kernel(const int64_t *total, int64_t cap, int *d_n, int *overflow) {
    const int64_t t = *total;
    const bool over = t > cap;
    *d_n = over ? 0 : (int)t;
    if (over) *overflow = 1;
}

void launch_clamp_count(const int64_t *total, int64_t cap, int *d_n, int *overflow, cudaStream_t st) {
    clamp_count_kernel<<<1, 1, 0, st>>>(total, cap, d_n, overflow);
}

}  // namespace msplat
