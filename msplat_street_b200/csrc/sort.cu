// Tile-intersection binning: exclusive scan, depth order, key emission, stable LSD
// radix sort and tile ranges.
//
// The reference builds per-tile lists ordered by (depth bits, Gaussian index)
// (bin_and_sort, core/cpu/msplat_cpu.cpp:505-567). Here the visible Gaussians are
// sorted by depth bits once (stable, so ties keep index order); every (Gaussian, tile)
// pair is then emitted in that order at offsets from an exclusive scan of
// tiles-per-Gaussian, keyed by its tile id alone. A STABLE radix sort over the
// ceil(log2 tiles) tile bits then yields, within each tile, ascending depth with ties
// in Gaussian order -- exactly the reference's order -- without a per-tile sort or any
// cap on a tile's list. The sort carries the emission index as its value; the map
// kernel turns it into the Gaussian id per sorted slot and the inverse permutation
// that the backward pass uses to reduce per-Gaussian gradients deterministically.
//
// The radix sort is reduce-then-scan per 8-bit digit: a histogram kernel, a device
// scan of the digit-major counts, and a scatter kernel that ranks keys stably inside
// each 2048-key block with warp match/popc. No block waits on another block.
#include <algorithm>
#include <atomic>

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

// Small inputs: one 1024-thread block walks the array in chunks of 4096 with a
// running carry (one launch instead of three).
constexpr int SCAN_SMALL = 16384, SMALL_ITEMS = 4;

template <typename TO>
__global__ void __launch_bounds__(1024) scan_small_kernel(const int32_t *in, int n, TO *out, TO *total) {
    __shared__ TO ws[33];
    TO carry = 0;
    for (int base = 0; base < n; base += 1024 * SMALL_ITEMS) {
        const int i0 = base + threadIdx.x * SMALL_ITEMS;
        TO v[SMALL_ITEMS], s = 0;
#pragma unroll
        for (int j = 0; j < SMALL_ITEMS; j++) {
            v[j] = i0 + j < n ? (TO)in[i0 + j] : TO(0);
            s += v[j];
        }
        TO tot;
        TO ex = block_exclusive_scan<TO>(s, ws, tot) + carry;
#pragma unroll
        for (int j = 0; j < SMALL_ITEMS; j++) {
            if (i0 + j < n) out[i0 + j] = ex;
            ex += v[j];
        }
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <typename TO>
void scan_exclusive(const int32_t *in, TO *out, int n, TO *d_total, TO *partials, cudaStream_t st) {
    if (n <= 0) {
        if (d_total) cudaMemsetAsync(d_total, 0, sizeof(TO), st);
        return;
    }
    if (n <= SCAN_SMALL) {
        scan_small_kernel<TO><<<1, 1024, 0, st>>>(in, n, out, d_total);
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
// Depth order and key emission.
//
// The reference orders each tile's list by (depth bits, Gaussian index). Here the
// Gaussians are first sorted by depth bits, stably (ties keep index order), and each
// one's intersections are emitted at offsets from a scan of tile counts taken in that
// order; a stable sort of the emitted entries by tile id alone then leaves every tile's
// entries in (depth, index) order. The per-intersection sort needs only ceil(log2
// tiles) key bits (2 passes up to 65,536 tiles) instead of 32 more depth bits.

// Depth keys: the float bits of the depth, which for the positive depths of visible
// Gaussians order like the numbers; Gaussians with no tiles go last.
__global__ void depth_keys_kernel(int n, const Splat *splats, const int32_t *n_tiles, uint32_t *keys, uint32_t *vals) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = n_tiles[i] > 0 ? __float_as_uint(splats[i].depth) : 0xffffffffu;
    vals[i] = (uint32_t)i;
}

__global__ void gather_counts_kernel(int n, const uint32_t *order, const int32_t *n_tiles, int32_t *cnt) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) cnt[r] = n_tiles[order[r]];
}

__global__ void scatter_offsets_kernel(int n, const uint32_t *order, const int64_t *off_sorted, int64_t *offsets) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r < n) offsets[order[r]] = off_sorted[r];
}

void launch_depth_offsets(int n, const Splat *splats, const int32_t *n_tiles, DepthScratch &s, int64_t *offsets,
                          int64_t *d_total, int64_t *scan_part, cudaStream_t st) {
    if (n <= 0) {
        cudaMemsetAsync(d_total, 0, sizeof(int64_t), st);
        return;
    }
    const int nb = (n + 255) / 256;
    depth_keys_kernel<<<nb, 256, 0, st>>>(n, splats, n_tiles, s.keys[0], s.vals[0]);
    const int cur = radix_sort_pairs32(s.keys, s.vals, n, 32, s.radix_scratch, st);
    if (cur != 0)  // four 8-bit passes end in buffer 0; emission reads the order there
        cudaMemcpyAsync(s.vals[0], s.vals[1], (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    gather_counts_kernel<<<nb, 256, 0, st>>>(n, s.vals[cur], n_tiles, s.counts);
    scan_exclusive<int64_t>(s.counts, s.off_sorted, n, d_total, scan_part, st);
    scatter_offsets_kernel<<<nb, 256, 0, st>>>(n, s.vals[cur], s.off_sorted, offsets);
}

__device__ __forceinline__ void rect_of(const Splat &s, float ax, float ay, int tx, int ty, int &x0, int &y0, int &x1,
                                        int &y1) {
    float ccx = s.x / (float)TILE, ccy = s.y / (float)TILE;
    float rrx = ax / (float)TILE, rry = ay / (float)TILE;
    x0 = min(max(0, (int)(ccx - rrx)), tx);
    x1 = min(max(0, (int)(ccx + rrx + 1)), tx);
    y0 = min(max(0, (int)(ccy - rry)), ty);
    y1 = min(max(0, (int)(ccy + rry + 1)), ty);
}

// Emission of each Gaussian's intersections: the tiles of its rectangle [x0, x1) x
// [y0, y1) in row-major order at emission indices e0, e0 + 1, ..., key = base + tile
// id, value = emission index (or, with emit_gid null -- render-only frames with no
// backward -- the Gaussian id itself, so the sorted values are the per-intersection
// ids with no gather). cap: buffer capacity (entries at or past it are dropped).
// Rectangles of up to SMALL_RECT tiles are written by their own thread; larger ones by
// the whole warp, lane l writing entries l, l + 32, ..., so their stores coalesce.
//
// Two thread-to-Gaussian maps, the same entries either way. BY_DEPTH: thread j takes
// the Gaussian at position j of the depth order; the emission offsets follow that
// order, so neighbouring threads write neighbouring ranges and stores fill whole
// sectors between them -- the better map when most Gaussians cover a few tiles each
// (renders of large scenes). By index: thread i takes Gaussian i; near-camera
// Gaussians with hundreds of tiles, which sit side by side in the depth order, then
// spread over many warps instead of falling to a few warps one after another -- the
// better map for training views, where such Gaussians carry much of the work.
constexpr int SMALL_RECT = 8;

__device__ __forceinline__ void emit_one(int64_t e, uint32_t key, int gid, uint32_t *keys, uint32_t *vals,
                                         int32_t *emit_gid) {
    keys[e] = key;
    if (emit_gid) {
        vals[e] = (uint32_t)e;
        emit_gid[e] = gid;
    } else {
        vals[e] = (uint32_t)gid;
    }
}

// Every lane of the warp must call it.
__device__ __forceinline__ void emit_rect(bool ok, int x0, int y0, int x1, int y1, int tiles_x, uint32_t base,
                                          int64_t e0, int gid, int64_t cap, uint32_t *keys, uint32_t *vals,
                                          int32_t *emit_gid) {
    const int w = x1 - x0, cnt = ok ? w * (y1 - y0) : 0;
    if (cnt > 0 && cnt <= SMALL_RECT) {
        int64_t e = e0;
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1 && e < cap; x++, e++)
                emit_one(e, base + (uint32_t)(y * tiles_x + x), gid, keys, vals, emit_gid);
    }
    unsigned big = __ballot_sync(0xffffffffu, cnt > SMALL_RECT);
    const int lane = threadIdx.x & 31;
    while (big) {  // warp-uniform
        const int src = __ffs(big) - 1;
        big &= big - 1;
        const int sw = __shfl_sync(0xffffffffu, w, src), sc = __shfl_sync(0xffffffffu, cnt, src);
        const int sx0 = __shfl_sync(0xffffffffu, x0, src), sy0 = __shfl_sync(0xffffffffu, y0, src);
        const int stx = __shfl_sync(0xffffffffu, tiles_x, src), sg = __shfl_sync(0xffffffffu, gid, src);
        const uint32_t sb = __shfl_sync(0xffffffffu, base, src);
        const int64_t se = __shfl_sync(0xffffffffu, (long long)e0, src);
        for (int j = lane; j < sc; j += 32) {
            const int64_t e = se + j;
            if (e >= cap) break;
            emit_one(e, sb + (uint32_t)((sy0 + j / sw) * stx + sx0 + j % sw), sg, keys, vals, emit_gid);
        }
    }
}

struct EmitSrc {
    const int32_t *n_tiles;      // per Gaussian (index map)
    const int64_t *offsets;      // per Gaussian (index map)
    const uint32_t *order;       // depth order (BY_DEPTH)
    const int32_t *cnt_sorted;   // tile counts in depth order (BY_DEPTH)
    const int64_t *off_sorted;   // emission offsets in depth order (BY_DEPTH)
};

// BATCH: instance g (a Gaussian of one view) keys its tiles with the view's first
// global tile added, so one stable sort orders every view's tiles at once and each
// tile's list is the one the single-view sort gives.
template <bool BATCH, bool BY_DEPTH>
__global__ void emit_keys_kernel(int n, const Splat *splats, const float *aabb, const EmitSrc src, int tiles_x,
                                 int tiles_y, const BatchDesc d, uint32_t *keys, uint32_t *vals, int32_t *emit_gid,
                                 int64_t cap) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = j < n && (BY_DEPTH ? src.cnt_sorted[j] : src.n_tiles[j]) > 0;
    int x0 = 0, y0 = 0, x1 = 0, y1 = 0, g = 0, tx = tiles_x;
    uint32_t base = 0;
    int64_t e0 = 0;
    if (ok) {
        g = BY_DEPTH ? (int)src.order[j] : j;
        int ty = tiles_y;
        if (BATCH) {
            const int v = find_view(d.inst_off, d.n_views, g);
            tx = d.tiles_x[v];
            ty = d.tiles_y[v];
            base = (uint32_t)d.tile_off[v];
        }
        rect_of(splats[g], aabb[2 * g], aabb[2 * g + 1], tx, ty, x0, y0, x1, y1);
        e0 = BY_DEPTH ? src.off_sorted[j] : src.offsets[g];
    }
    emit_rect(ok, x0, y0, x1, y1, tx, base, e0, g, cap, keys, vals, emit_gid);
}

namespace {
EmitSrc emit_src(const int32_t *n_tiles, const int64_t *offsets, const DepthScratch *ds) {
    EmitSrc s{n_tiles, offsets, nullptr, nullptr, nullptr};
    if (ds) {
        s.order = ds->vals[0];
        s.cnt_sorted = ds->counts;
        s.off_sorted = ds->off_sorted;
    }
    return s;
}
}  // namespace

void launch_emit_keys(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles, const int64_t *offsets,
                      int tiles_x, int tiles_y, uint32_t *keys, uint32_t *vals, int32_t *emit_gid, cudaStream_t st,
                      int64_t cap) {
    if (n <= 0 || cap <= 0) return;
    emit_keys_kernel<false, false><<<(n + 127) / 128, 128, 0, st>>>(
        n, splats, aabb, emit_src(n_tiles, offsets, nullptr), tiles_x, tiles_y, BatchDesc{}, keys, vals, emit_gid,
        cap);
}

void launch_emit_keys_batch(int n, const Splat *splats, const float *aabb, const int32_t *n_tiles,
                            const int64_t *offsets, const DepthScratch *ds, const BatchDesc &d, uint32_t *keys,
                            uint32_t *vals, int32_t *emit_gid, cudaStream_t st, int64_t cap) {
    if (n <= 0) return;
    const EmitSrc src = emit_src(n_tiles, offsets, ds);
    if (ds)
        emit_keys_kernel<true, true><<<(n + 127) / 128, 128, 0, st>>>(n, splats, aabb, src, 0, 0, d, keys, vals,
                                                                      emit_gid, cap);
    else
        emit_keys_kernel<true, false><<<(n + 127) / 128, 128, 0, st>>>(n, splats, aabb, src, 0, 0, d, keys, vals,
                                                                       emit_gid, cap);
}

// ---------------------------------------------------------------------------------
// Stable LSD radix sort of (key, u32 value) pairs by key bits [0, key_bits), for
// 32- and 64-bit keys.

constexpr int RADIX = 256;
// Keys per block: THREADS x ITEMS. Large sorts of 32-bit keys take 256 threads x 16
// items (4096 keys a block): each digit's run in a block then averages 16 entries, so
// the scatter's stores come in runs of 64 bytes or more, and the per-block digit counts
// (256 per block, scanned every pass) stay small next to the keys. Below LARGE_SORT
// keys, 256 x 8 (2048 keys a block) keeps enough blocks to fill the GPU; 64-bit keys
// take 2048-key blocks too (4096 would need 48 KB of staging per block). Measured and
// not kept: 512 x 8 and 1024 x 4 blocks for the large 32-bit sort (two and one blocks
// per SM: the 46 M-key tile sort of a 1080p frame 1.06 and 1.51 ms against 1.02), and
// the largest shared-memory carveout (1.06 ms: the scatter's loads and stores want
// the L1). The scatter is bound by its integer pipe (ALU 64 % of peak, issue 54 %):
// the ranking's ballots, not DRAM, set its pace.
constexpr int SORT_THREADS = 256;
constexpr int LARGE_SORT = 4 << 20;
constexpr int MAX_SORT_THREADS = 1024;

// Up to this many blocks (131,072 keys at 2048 a block, the depth order of a training
// view), each scatter block sums the per-block digit counts itself instead of a
// separate scan launch over them.
constexpr int DIRECT_SORT_BLOCKS = 64;

// The most blocks any sort of up to n keys uses (scratch sizing): 2048-key blocks,
// the smallest of every block shape below.
int radix_max_blocks(int n) { return (n + 2047) / 2048; }

// d_n (may be null): a device-side count that caps n (capacity-bounded launches)
// The lanes of the warp whose digit equals this lane's (d in 0..RADIX, RADIX marking
// a lane with no key): nine ballots, one per bit of d, each narrowing the set to the
// lanes that agree on that bit. Constant cost whatever the number of distinct digits
// in the warp (a warp of scattered tile ids holds up to 32).
// Only the bits a pass's digits can hold take a ballot (mask, uniform), and the no-key
// bit only in a block that is not full (full: every lane holds a key).
__device__ __forceinline__ unsigned digit_peers(int d, uint32_t mask, bool full) {
    unsigned m = 0xffffffffu;
#pragma unroll
    for (int b = 0; b < 9; b++) {
        if (b < 8 ? !((mask >> b) & 1u) : full) continue;  // uniform
        const bool on = (d >> b) & 1;
        const unsigned bal = __ballot_sync(0xffffffffu, on);
        m &= on ? bal : ~bal;
    }
    return m;
}

// Counting needs no ranks: each warp adds its keys' digits to its own shared-memory
// histogram with one atomic per key (lanes of a warp that share a digit are resolved
// by the shared-memory atomic unit), and the block sums the warps' histograms.
template <typename K, int THREADS, int SORT_ITEMS>
__global__ void __launch_bounds__(THREADS) radix_hist_kernel(const K *keys, int n, const int *d_n, int shift,
                                                             uint32_t mask, uint32_t *counts, int nb) {
    constexpr int WARPS = THREADS / 32;
    __shared__ uint32_t h[WARPS][RADIX];
    if (d_n) n = min(n, *d_n);
    for (int i = threadIdx.x; i < WARPS * RADIX; i += THREADS) (&h[0][0])[i] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    constexpr int SORT_TILE = THREADS * SORT_ITEMS;
    const int base = blockIdx.x * SORT_TILE;
    int dig[SORT_ITEMS];
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++) {  // independent loads first
        const int k = base + j * THREADS + threadIdx.x;
        dig[j] = k < n ? (int)((keys[k] >> shift) & mask) : RADIX;
    }
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; j++)
        if (dig[j] < RADIX) atomicAdd(&h[warp][dig[j]], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < RADIX; i += THREADS) {
        uint32_t s = 0;
#pragma unroll
        for (int w = 0; w < WARPS; w++) s += h[w][i];
        counts[(size_t)i * nb + blockIdx.x] = s;
    }
}

// offs: the exclusive digit-major scan of the per-block digit counts; or, with offs
// null (a sort of at most DIRECT_SORT_BLOCKS blocks), counts: the per-block digit counts
// themselves, from which each block forms its own digit starts (no scan launch).
// The 64-bit-key scatter is held to 64 registers, four resident blocks per SM (32 M
// pairs of 40 bits: 2.35 instead of 2.49 ms); the 32-bit ones to 128 (the depth order
// of a street view's 100 k Gaussians ran 10 % slower at 64).
template <typename K, int THREADS, int SORT_ITEMS>
__global__ void __launch_bounds__(THREADS, sizeof(K) == 8 ? 1024 / THREADS : 512 / THREADS) radix_scatter_kernel(const K *kin, const uint32_t *vin, K *kout,
                                                                uint32_t *vout, int n, const int *d_n, int shift,
                                                                uint32_t mask, const int32_t *offs,
                                                                const uint32_t *counts, int nb) {
    // The block's keys are first ranked and placed in shared memory in digit order
    // (a block-local stable multisplit), then written out so that consecutive threads
    // write consecutive entries of each digit's run: coalesced global stores.
    static_assert(THREADS >= RADIX && THREADS <= MAX_SORT_THREADS, "a thread per digit");
    constexpr int WARPS = THREADS / 32;
    __shared__ uint32_t wcnt[WARPS][RADIX];
    __shared__ uint32_t gbase[RADIX], bstart[RADIX + 1];
    constexpr int SORT_TILE = THREADS * SORT_ITEMS;  // keys per block
    constexpr int WARP_KEYS = SORT_TILE / WARPS;     // contiguous keys per warp
    __shared__ uint32_t ws[33];
    extern __shared__ __align__(16) unsigned char sort_smem[];  // radix_scatter_smem<K, SORT_ITEMS>()
    K *skey = reinterpret_cast<K *>(sort_smem);
    uint32_t *sval = reinterpret_cast<uint32_t *>(skey + SORT_TILE);
    if (d_n) n = min(n, *d_n);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < WARPS * RADIX; i += THREADS) (&wcnt[0][0])[i] = 0;
    if (offs) {
        for (int i = threadIdx.x; i < RADIX; i += THREADS) gbase[i] = (uint32_t)offs[(size_t)i * nb + blockIdx.x];
    } else {  // thread d: digit d's count over all blocks and over the blocks before this one
        uint32_t tot = 0u, before = 0u;
        if (threadIdx.x < RADIX) {
            const uint32_t *row = counts + (size_t)threadIdx.x * nb;
            for (int b = 0; b < nb; b++) {
                const uint32_t c = row[b];
                tot += c;
                if (b < (int)blockIdx.x) before += c;
            }
        }
        uint32_t all;
        const uint32_t ex = block_exclusive_scan<uint32_t>(tot, ws, all) + before;
        if (threadIdx.x < RADIX) gbase[threadIdx.x] = ex;
    }
    K key[SORT_ITEMS];
    uint32_t val[SORT_ITEMS], rank[SORT_ITEMS];
    int dig[SORT_ITEMS];
    const int base = blockIdx.x * SORT_TILE + warp * WARP_KEYS;
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {  // independent loads first
        const int k = base + r * 32 + lane;
        const bool ok = k < n;
        key[r] = ok ? kin[k] : K(0);
        val[r] = ok ? vin[k] : 0u;
        dig[r] = ok ? (int)((key[r] >> shift) & mask) : RADIX;
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const bool full = (int64_t)blockIdx.x * SORT_TILE + SORT_TILE <= (int64_t)n;
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {
        const int d = dig[r];
        const bool ok = d < RADIX;
        const unsigned peers = digit_peers(d, mask, full);
        const uint32_t before = ok ? wcnt[warp][d] : 0u;
        rank[r] = before + (uint32_t)__popc(peers & lt);
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) wcnt[warp][d] = before + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive prefix over warps, then over digits (block-local starts)
    uint32_t tot = 0;
    if (threadIdx.x < RADIX) {
        const int d = threadIdx.x;
#pragma unroll
        for (int w = 0; w < WARPS; w++) {
            const uint32_t t = wcnt[w][d];
            wcnt[w][d] = tot;
            tot += t;
        }
    }
    uint32_t btot;
    const uint32_t ex = block_exclusive_scan<uint32_t>(threadIdx.x < RADIX ? tot : 0u, ws, btot);
    if (threadIdx.x < RADIX) bstart[threadIdx.x] = ex;
    if (threadIdx.x == 0) bstart[RADIX] = btot;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SORT_ITEMS; r++) {
        const int d = dig[r];
        if (d < RADIX) {
            const uint32_t lp = bstart[d] + wcnt[warp][d] + rank[r];
            skey[lp] = key[r];
            sval[lp] = val[r];
        }
    }
    __syncthreads();
    const int valid = (int)bstart[RADIX];
    for (int i = threadIdx.x; i < valid; i += THREADS) {
        const K kk = skey[i];
        const int d = (int)((kk >> shift) & mask);
        const uint32_t pos = gbase[d] + ((uint32_t)i - bstart[d]);
        kout[pos] = kk;
        vout[pos] = sval[i];
    }
}

template <typename K, int THREADS, int ITEMS>
constexpr size_t radix_scatter_smem() {
    return (size_t)THREADS * ITEMS * (sizeof(K) + sizeof(uint32_t));
}

size_t radix_scratch_bytes(int n) {
    const int nb = radix_max_blocks(n > 1 ? n : 1);
    const size_t cnt = (size_t)RADIX * nb;
    return cnt * sizeof(int32_t) * 2 + (size_t)scan_blocks((int)cnt) * sizeof(int32_t) + 64;
}

// Sorts (k[0], v[0]) using (k[1], v[1]) as the ping-pong buffers; returns the index
// (0 or 1) of the buffer pair holding the result. With d_n, n is a capacity and the
// count is read on the device (no host round trip; every pass runs).
template <typename K, int THREADS, int ITEMS>
int radix_sort_impl(K *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st, const int *d_n) {
    const int nb = (n + THREADS * ITEMS - 1) / (THREADS * ITEMS);
    const size_t cnt = (size_t)RADIX * nb;
    int32_t *counts = reinterpret_cast<int32_t *>(scratch);
    int32_t *offs = counts + cnt;
    int32_t *partials = offs + cnt;
    constexpr size_t smem = radix_scatter_smem<K, THREADS, ITEMS>();
    {  // once per device: the dynamic staging (with the static arrays it can pass the 48 KB
       // default)
        static std::atomic<uint64_t> done{0};
        int dev = 0;
        cudaGetDevice(&dev);
        const uint64_t bit = 1ull << (dev & 63);
        if (!(done.load() & bit)) {
            cudaFuncSetAttribute(radix_scatter_kernel<K, THREADS, ITEMS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem);
            done.fetch_or(bit);
        }
    }
    int cur = 0;
    for (int shift = 0; shift < key_bits; shift += 8) {
        const int bits = key_bits - shift < 8 ? key_bits - shift : 8;  // digits above key_bits are ignored
        const uint32_t mask = (1u << bits) - 1u;
        radix_hist_kernel<K, THREADS, ITEMS><<<nb, THREADS, 0, st>>>(k[cur], n, d_n, shift, mask,
                                                                     reinterpret_cast<uint32_t *>(counts), nb);
        const bool direct = nb <= DIRECT_SORT_BLOCKS;
        if (!direct) scan_exclusive<int32_t>(counts, offs, (int)cnt, nullptr, partials, st);
        radix_scatter_kernel<K, THREADS, ITEMS><<<nb, THREADS, smem, st>>>(
            k[cur], v[cur], k[cur ^ 1], v[cur ^ 1], n, d_n, shift, mask, direct ? nullptr : offs,
            reinterpret_cast<const uint32_t *>(counts), nb);
        cur ^= 1;
    }
    return cur;
}

template <typename K>
int radix_sort_dispatch(K *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st, const int *d_n) {
    if ((!d_n && n <= 1) || n <= 0 || key_bits <= 0) return 0;
    if constexpr (sizeof(K) == 4) {
        if (n >= LARGE_SORT) return radix_sort_impl<K, 256, 16>(k, v, n, key_bits, scratch, st, d_n);
    }
    return radix_sort_impl<K, 256, 8>(k, v, n, key_bits, scratch, st, d_n);
}

int radix_sort_pairs(uint64_t *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st,
                     const int *d_n) {
    return radix_sort_dispatch<uint64_t>(k, v, n, key_bits, scratch, st, d_n);
}

int radix_sort_pairs32(uint32_t *k[2], uint32_t *v[2], int n, int key_bits, void *scratch, cudaStream_t st,
                       const int *d_n) {
    return radix_sort_dispatch<uint32_t>(k, v, n, std::min(key_bits, 32), scratch, st, d_n);
}

// ---------------------------------------------------------------------------------
// Tile ranges by binary search over the sorted tile ids (empty tiles get start ==
// end == the running count, as the reference's prefix sums give), and the per-slot
// Gaussian id / inverse map.

__global__ void tile_ranges_kernel(const uint32_t *keys, int n, int T, int32_t *tile_start, int32_t *tile_end,
                                   const int *d_n, const int *d_T) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_n) n = min(n, *d_n);
    if (d_T) T = min(T, *d_T);
    if (t > T) return;
    int lo = 0, hi = n;  // first position whose tile id >= t
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((int)keys[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    if (t < T) tile_start[t] = lo;
    if (t > 0) tile_end[t - 1] = lo;
}

// inv (may be null, render-only frames): emission index -> sorted position, for the
// backward's per-Gaussian reduction
__global__ void isect_map_kernel(const uint32_t *sorted_e, int n, const int32_t *emit_gid, int32_t *isect_gid,
                                 int32_t *inv, const int *d_n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (d_n) n = min(n, *d_n);
    if (k >= n) return;
    const uint32_t e = sorted_e[k];
    isect_gid[k] = emit_gid[e];
    if (inv) inv[e] = k;
}

void launch_tile_ranges(const uint32_t *keys, int n, int T, int32_t *tile_start, int32_t *tile_end, cudaStream_t st,
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
