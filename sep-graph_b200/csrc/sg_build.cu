// GPU graph construction.
//
// Two host-side steps of the reference run here on the device:
//  * csr_tocsc (include/groute/graphs/csr_graph.h:329-397), the CSR -> CSC
//    transpose behind every pull variant.  The reference's loop is a stable
//    counting sort of the edges by destination: each in-edge list comes out
//    ordered by source and, among parallel edges, by CSR position.
//  * the edge-list preprocessing of samples/tools/gtools.cpp:56-328
//    (--deself_cycle, --deduplicate, --d2ud), fused with the CSR build of the
//    edge list itself.
// Both are counting sorts: per-row counts (atomics), an exclusive scan into
// row offsets, a scatter whose order inside a row is arbitrary, then a
// segmented sort of every row by a key that is unique per entry (it holds the
// entry's input position), so the result never depends on the scatter order.
//
// Segmented sort: rows of 2-32 keys are sorted by one warp in registers
// (bitonic network over shuffles), rows up to 4096 keys by one block in shared
// memory (bitonic), longer rows in 4096-key chunks followed by merge-path
// passes that double the sorted run length, ping-ponging with a compact
// temporary.  All of it is integer work bounded by HBM and L2 bandwidth.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <vector>

#include "sg_runtime.cuh"

namespace sgb {
namespace gbuild {

using sepgraph::dev::kFullMask;

constexpr uint32_t kWarpKeys = 256;    // rows up to this many keys sort in one warp's registers
constexpr uint32_t kSmemKeys = 4096;   // rows up to this many keys sort in shared memory
constexpr uint32_t kSortThreads = 256;
constexpr uint32_t kMergeItems = kSmemKeys / kSortThreads;  // outputs per thread in a merge pass
constexpr uint32_t kScanThreads = 1024;
constexpr uint32_t kScanItems = 4;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
constexpr uint32_t kScanMaxParts = 2 * kScanThreads;  // partial sums one block scans
constexpr uint64_t kMaxEntries = 0xfffffffeull;          // entries must index with uint32

template <class K>
__device__ __forceinline__ K key_max() {
    return (K)~(K)0;
}

// Temporary device buffers of one call, named in the context's grow-only
// scratch (released by sg_ctx_release_cached): repeated builds and
// transposes reuse them instead of allocating and freeing every time.  Each
// call site has its own prefix and each allocation of a Tmp its own number,
// so buffers whose lifetimes overlap never share a name; a later call with
// the same prefix reuses the buffers of an earlier one, which is finished by
// then (all work of a context is ordered on its stream).
struct Tmp {
    sg_ctx *ctx;
    const char *prefix;
    unsigned n = 0;
    Tmp(sg_ctx *c, const char *p) : ctx(c), prefix(p) {}
    template <class T>
    cudaError_t alloc(T **p, uint64_t count) {
        char name[48];
        std::snprintf(name, sizeof name, "gb_%s_%u", prefix, n++);
        if (!ctx->graph_ws) ctx->graph_ws = new Workspace(&ctx->stream, device_pool(ctx->device));
        return ctx->graph_ws->get(name, (size_t)std::max<uint64_t>(count, 1), p);
    }
};

inline unsigned grid_for(uint64_t work, unsigned per_block, unsigned cap = 148 * 16) {
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((work + per_block - 1) / per_block, cap));
}

// ------------------------------------------------------------------ exclusive scan
// out[i] = sum of in[0..i) for i <= n, in three launches: per-block sums of
// contiguous ranges, one block scanning those sums, then each block scanning
// its range in tiles with a running carry.  *total receives the full sum (64
// bits, so the caller can reject offsets that overflow uint32).

__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long x, unsigned long long *warp_sums,
                                                                   unsigned long long *block_total) {
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    unsigned long long inc = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(kFullMask, inc, d);
        if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31) warp_sums[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        unsigned long long v = lane < nwarps ? warp_sums[lane] : 0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFullMask, v, d);
            if (lane >= (uint32_t)d) v += y;
        }
        warp_sums[lane] = v;
    }
    __syncthreads();
    *block_total = warp_sums[nwarps - 1];
    const unsigned long long r = inc - x + (wid ? warp_sums[wid - 1] : 0);
    __syncthreads();
    return r;
}

__global__ void scan_reduce_kernel(const uint32_t *in, uint64_t n, uint64_t per, unsigned long long *part) {
    __shared__ unsigned long long ws[32];
    const uint64_t lo = blockIdx.x * per, hi = min(n, lo + per);
    unsigned long long s = 0;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += in[i];
    unsigned long long total;
    block_exclusive_scan(s, ws, &total);
    if (threadIdx.x == 0) part[blockIdx.x] = total;
}

__global__ void scan_parts_kernel(unsigned long long *part, uint32_t nparts, unsigned long long *total) {
    __shared__ unsigned long long ws[32];
    const uint32_t i0 = 2 * threadIdx.x, i1 = i0 + 1;
    const unsigned long long a = i0 < nparts ? part[i0] : 0, b = i1 < nparts ? part[i1] : 0;
    unsigned long long t;
    const unsigned long long ex = block_exclusive_scan(a + b, ws, &t);
    if (i0 < nparts) part[i0] = ex;
    if (i1 < nparts) part[i1] = ex + a;
    if (threadIdx.x == 0) *total = t;
}

__global__ void scan_apply_kernel(const uint32_t *in, uint64_t n, uint64_t per, const unsigned long long *part,
                                  const unsigned long long *total, uint32_t *out) {
    __shared__ unsigned long long ws[32];
    const uint64_t lo = blockIdx.x * per, hi = min(n, lo + per);
    unsigned long long carry = part[blockIdx.x];
    for (uint64_t t0 = lo; t0 < hi; t0 += kScanTile) {
        const uint64_t i0 = t0 + (uint64_t)threadIdx.x * kScanItems;
        uint32_t v[kScanItems];
        unsigned long long s = 0;
#pragma unroll
        for (uint32_t k = 0; k < kScanItems; ++k) {
            v[k] = i0 + k < hi ? in[i0 + k] : 0u;
            s += v[k];
        }
        unsigned long long tile_total;
        unsigned long long run = carry + block_exclusive_scan(s, ws, &tile_total);
#pragma unroll
        for (uint32_t k = 0; k < kScanItems; ++k) {
            if (i0 + k < hi) out[i0 + k] = (uint32_t)run;
            run += v[k];
        }
        carry += tile_total;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = (uint32_t)*total;
}

// Exclusive scan of n counts into out[0..n]; *total_host gets the sum.
sg_status exclusive_scan(sg_ctx *ctx, Tmp &tmp, const uint32_t *in, uint64_t n, uint32_t *out,
                         unsigned long long *total_host) {
    const cudaStream_t s = ctx->stream;
    const uint32_t nparts = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(kScanMaxParts, (n + kScanTile - 1) / kScanTile));
    const uint64_t per = std::max<uint64_t>(1, (n + nparts - 1) / nparts);
    unsigned long long *part, *total;
    SG_TRY_CUDA(ctx, tmp.alloc(&part, nparts + 1));
    total = part + nparts;
    scan_reduce_kernel<<<nparts, kScanThreads, 0, s>>>(in, n, per, part);
    scan_parts_kernel<<<1, kScanThreads, 0, s>>>(part, nparts, total);
    scan_apply_kernel<<<nparts, kScanThreads, 0, s>>>(in, n, per, part, total, out);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(total_host, total, sizeof *total, cudaMemcpyDeviceToHost, s));
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    return SG_OK;
}

// ------------------------------------------------------------------ segmented sort

template <class K>
__device__ __forceinline__ K warp_bitonic(K x, uint32_t lane) {
#pragma unroll
    for (uint32_t k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const K y = __shfl_xor_sync(kFullMask, x, j);
            const bool up = (lane & k) == 0, lower = (lane & j) == 0;
            x = (lower == up) ? (x < y ? x : y) : (x < y ? y : x);
        }
    }
    return x;
}

// Bitonic sort of 32*E keys held striped across a warp (element r*32+lane in
// register r): exchanges at distance >= 32 swap registers within a lane,
// shorter ones go through shuffles.
template <class K, int E>
__device__ __forceinline__ void warp_bitonic_regs(K (&x)[E], uint32_t lane) {
#pragma unroll
    for (uint32_t k = 2; k <= 32u * E; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const uint32_t jr = j >> 5;
#pragma unroll
                for (uint32_t r = 0; r < (uint32_t)E; ++r) {
                    if ((r & jr) == 0) {
                        const uint32_t r2 = r | jr;
                        const bool asc = ((r * 32 + lane) & k) == 0;
                        const K a = x[r], b = x[r2];
                        const bool swap = (a > b) == asc;
                        x[r] = swap ? b : a;
                        x[r2] = swap ? a : b;
                    }
                }
            } else {
#pragma unroll
                for (uint32_t r = 0; r < (uint32_t)E; ++r) {
                    const K y = __shfl_xor_sync(kFullMask, x[r], j);
                    const bool asc = ((r * 32 + lane) & k) == 0, lower = (lane & j) == 0;
                    x[r] = (lower == asc) ? (x[r] < y ? x[r] : y) : (x[r] < y ? y : x[r]);
                }
            }
        }
    }
}

template <class K, int E>
__device__ __forceinline__ void warp_sort_row(K *keys, uint32_t b, uint32_t len, uint32_t lane) {
    K x[E];
#pragma unroll
    for (uint32_t r = 0; r < (uint32_t)E; ++r) {
        const uint32_t i = r * 32 + lane;
        x[r] = i < len ? keys[b + i] : key_max<K>();
    }
    warp_bitonic_regs<K, E>(x, lane);
#pragma unroll
    for (uint32_t r = 0; r < (uint32_t)E; ++r) {
        const uint32_t i = r * 32 + lane;
        if (i < len) keys[b + i] = x[r];
    }
}

// One warp per listed row of 33-256 keys.
template <class K>
__global__ void sort_rows_warp_kernel(const uint2 *segs, const uint32_t *count_dev, uint32_t cap, K *keys) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = min(*count_dev, cap);
    for (uint32_t i = gw; i < n; i += nw) {
        const uint2 sg = segs[i];
        if (sg.y <= 64) warp_sort_row<K, 2>(keys, sg.x, sg.y, lane);
        else if (sg.y <= 128) warp_sort_row<K, 4>(keys, sg.x, sg.y, lane);
        else warp_sort_row<K, 8>(keys, sg.x, sg.y, lane);
    }
}

// One warp per 32 rows: rows of 2-32 keys are sorted in place; longer rows are
// listed (begin, length) for the one-warp sort (up to kWarpKeys), the
// shared-memory sort (up to kSmemKeys) or the chunked merge sort.
template <class K>
__global__ void sort_rows_small_kernel(const uint32_t *off, uint32_t nv, K *keys, uint2 *wrows, uint32_t wrows_cap,
                                       uint2 *mid, uint32_t mid_cap, uint2 *big, uint32_t big_cap, uint32_t *counts) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t base = gw * 32; base < nv; base += nw * 32) {
        const uint64_t v = base + lane;
        uint32_t b = 0, len = 0;
        if (v < nv) {
            b = off[v];
            len = off[v + 1] - b;
        }
        if (len > 32) {
            if (len <= kWarpKeys) {
                const uint32_t p = atomicAdd(counts + 2, 1u);
                if (p < wrows_cap) wrows[p] = make_uint2(b, len);
            } else if (len <= kSmemKeys) {
                const uint32_t p = atomicAdd(counts, 1u);
                if (p < mid_cap) mid[p] = make_uint2(b, len);
            } else {
                const uint32_t p = atomicAdd(counts + 1, 1u);
                if (p < big_cap) big[p] = make_uint2(b, len);
            }
        }
        uint32_t m = __ballot_sync(kFullMask, len >= 2 && len <= 32);
        while (m) {
            const uint32_t j = __ffs(m) - 1;
            m &= m - 1;
            const uint32_t bj = __shfl_sync(kFullMask, b, j), lj = __shfl_sync(kFullMask, len, j);
            K x = lane < lj ? keys[bj + lane] : key_max<K>();
            x = warp_bitonic(x, lane);
            if (lane < lj) keys[bj + lane] = x;
        }
    }
}

// One block per segment of at most kSmemKeys keys: bitonic sort in shared
// memory over the segment padded to a power of two.  The segment count is
// read from device memory (count_dev) or given (count_dev == nullptr).
template <class K>
__global__ void __launch_bounds__(kSortThreads) sort_segments_kernel(const uint2 *segs, const uint32_t *count_dev,
                                                                    uint32_t count, K *keys) {
    __shared__ K sk[kSmemKeys];
    const uint32_t n = count_dev ? min(*count_dev, count) : count;
    for (uint32_t sgi = blockIdx.x; sgi < n; sgi += gridDim.x) {
        const uint2 sg = segs[sgi];
        uint32_t n2 = 2;
        while (n2 < sg.y) n2 <<= 1;
        for (uint32_t i = threadIdx.x; i < n2; i += blockDim.x) sk[i] = i < sg.y ? keys[sg.x + i] : key_max<K>();
        __syncthreads();
        for (uint32_t k = 2; k <= n2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < (n2 >> 1); i += blockDim.x) {
                    const uint32_t lo = ((i & ~(j - 1)) << 1) | (i & (j - 1)), hi = lo + j;
                    const K a = sk[lo], b = sk[hi];
                    if ((a > b) == ((lo & k) == 0)) {
                        sk[lo] = b;
                        sk[hi] = a;
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < sg.y; i += blockDim.x) keys[sg.x + i] = sk[i];
        __syncthreads();
    }
}

// Merge-path pass over the long rows: tile t = (base in keys, row length,
// offset of the tile in the row, base in the temporary) covers kSmemKeys
// outputs of the pair of sorted runs of length `run` that contains it.  Keys
// are unique, so the merge needs no tie rule.
template <class K>
__global__ void __launch_bounds__(kSortThreads) merge_pass_kernel(const uint4 *tiles, uint32_t ntiles, K *keys, K *tmp,
                                                                 uint32_t run, int to_tmp) {
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint4 tl = tiles[t];
        const K *src = to_tmp ? keys + tl.x : tmp + tl.w;
        K *dst = to_tmp ? tmp + tl.w : keys + tl.x;
        const uint32_t len = tl.y;
        const uint64_t run2 = 2ull * run;
        const uint32_t pair = (uint32_t)(tl.z / run2 * run2);
        const uint32_t a1 = (uint32_t)min((uint64_t)pair + run, (uint64_t)len);
        const uint32_t b1 = (uint32_t)min((uint64_t)pair + run2, (uint64_t)len);
        const uint32_t la = a1 - pair, lb = b1 - a1;
        const K *A = src + pair, *B = src + a1;
        const uint32_t d = tl.z - pair + threadIdx.x * kMergeItems;
        if (d >= la + lb) continue;
        const uint32_t cnt = min(kMergeItems, la + lb - d);
        uint32_t lo = d > lb ? d - lb : 0, hi = min(d, la);
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (A[mid] < B[d - 1 - mid]) lo = mid + 1;
            else hi = mid;
        }
        uint32_t i = lo, j = d - lo;
        for (uint32_t k = 0; k < cnt; ++k) {
            const bool take_a = j >= lb || (i < la && A[i] < B[j]);
            dst[pair + d + k] = take_a ? A[i++] : B[j++];
        }
    }
}

template <class K>
__global__ void copy_tiles_kernel(const uint4 *tiles, uint32_t ntiles, K *keys, const K *tmp) {
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint4 tl = tiles[t];
        const uint32_t end = min(tl.z + kSmemKeys, tl.y);
        for (uint32_t i = tl.z + threadIdx.x; i < end; i += blockDim.x) keys[tl.x + i] = tmp[tl.w + i];
    }
}

// Sorts every row [off[v], off[v+1]) of keys ascending.  Keys must be unique
// within a row.
template <class K>
sg_status sort_rows(sg_ctx *ctx, const uint32_t *off, uint32_t nv, uint64_t n, K *keys) {
    if (n < 2) return SG_OK;
    const cudaStream_t s = ctx->stream;
    Tmp tmp(ctx, "sort");
    const uint32_t wrows_cap = (uint32_t)(n / 33 + 1), mid_cap = (uint32_t)(n / (kWarpKeys + 1) + 1);
    const uint32_t big_cap = (uint32_t)(n / (kSmemKeys + 1) + 1);
    uint2 *wrows, *mid, *big;
    uint32_t *counts;  // [mid, big, warp rows]
    SG_TRY_CUDA(ctx, tmp.alloc(&wrows, wrows_cap));
    SG_TRY_CUDA(ctx, tmp.alloc(&mid, mid_cap));
    SG_TRY_CUDA(ctx, tmp.alloc(&big, big_cap));
    SG_TRY_CUDA(ctx, tmp.alloc(&counts, 3));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(counts, 0, 3 * sizeof(uint32_t), s));
    sort_rows_small_kernel<K><<<grid_for((uint64_t)nv, 256), 256, 0, s>>>(off, nv, keys, wrows, wrows_cap, mid, mid_cap,
                                                                        big, big_cap, counts);
    sort_rows_warp_kernel<K><<<148 * 8, 256, 0, s>>>(wrows, counts + 2, wrows_cap, keys);
    sort_segments_kernel<K><<<148 * 8, kSortThreads, 0, s>>>(mid, counts, mid_cap, keys);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    uint32_t hc[3];
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(hc, counts, sizeof hc, cudaMemcpyDeviceToHost, s));
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    const uint32_t nbig = std::min(hc[1], big_cap);
    if (!nbig) return SG_OK;
    std::vector<uint2> hb(nbig);
    SG_TRY_CUDA(ctx, cudaMemcpy(hb.data(), big, nbig * sizeof(uint2), cudaMemcpyDeviceToHost));
    std::sort(hb.begin(), hb.end(), [](uint2 a, uint2 b) { return a.x < b.x; });  // deterministic layout
    std::vector<uint2> chunks;
    std::vector<uint4> tiles;
    uint64_t tmp_len = 0;
    uint32_t max_len = 0;
    for (const uint2 &r : hb) {
        for (uint32_t c = 0; c < r.y; c += kSmemKeys) {
            chunks.push_back(make_uint2(r.x + c, std::min(kSmemKeys, r.y - c)));
            tiles.push_back(make_uint4(r.x, r.y, c, (uint32_t)tmp_len));
        }
        tmp_len += r.y;
        max_len = std::max(max_len, r.y);
    }
    uint2 *dchunks;
    uint4 *dtiles;
    K *ktmp;
    SG_TRY_CUDA(ctx, tmp.alloc(&dchunks, chunks.size()));
    SG_TRY_CUDA(ctx, tmp.alloc(&dtiles, tiles.size()));
    SG_TRY_CUDA(ctx, tmp.alloc(&ktmp, tmp_len));
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(dchunks, chunks.data(), chunks.size() * sizeof(uint2), cudaMemcpyHostToDevice, s));
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(dtiles, tiles.data(), tiles.size() * sizeof(uint4), cudaMemcpyHostToDevice, s));
    const uint32_t nt = (uint32_t)tiles.size();
    const unsigned grid = std::min<unsigned>(nt, 148 * 8);
    sort_segments_kernel<K><<<grid, kSortThreads, 0, s>>>(dchunks, nullptr, (uint32_t)chunks.size(), keys);
    int to_tmp = 1;
    for (uint64_t run = kSmemKeys; run < max_len; run <<= 1) {
        merge_pass_kernel<K><<<grid, kSortThreads, 0, s>>>(dtiles, nt, keys, ktmp, (uint32_t)run, to_tmp);
        to_tmp ^= 1;
    }
    if (!to_tmp) copy_tiles_kernel<K><<<grid, kSortThreads, 0, s>>>(dtiles, nt, keys, ktmp);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    return SG_OK;
}

// ------------------------------------------------------------------ CSR -> CSC

__global__ void count_by_col_kernel(const uint32_t *col, uint64_t ne, uint32_t *cnt) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < ne; e += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(cnt + __ldg(col + e), 1u);
}

__global__ void scatter_by_col_kernel(const uint32_t *col, uint64_t ne, uint32_t *cur, uint32_t *ekeys) {
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < ne; e += (uint64_t)gridDim.x * blockDim.x)
        ekeys[atomicAdd(cur + __ldg(col + e), 1u)] = (uint32_t)e;
}

// In-edge list entry p holds CSR edge index e; replace it by e's source
// (the row whose range holds e) and copy e's weight.
__global__ void csc_finish_kernel(const uint32_t *row, uint32_t nv, const uint32_t *w, uint64_t ne, uint32_t *ccol,
                                  uint32_t *cw) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < ne; p += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t e = ccol[p];
        uint32_t lo = 0, hi = nv;  // largest u with row[u] <= e
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldg(row + mid) <= e) lo = mid;
            else hi = mid - 1;
        }
        ccol[p] = lo;
        if (w) cw[p] = __ldg(w + e);
    }
}

__global__ void compare_csr_kernel(const uint32_t *ra, const uint32_t *rb, uint32_t nv, const uint32_t *ca,
                                   const uint32_t *cb, const uint32_t *wa, const uint32_t *wb, uint64_t ne,
                                   uint32_t *diff /* [structure, weights] */) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x, nt = (uint64_t)gridDim.x * blockDim.x;
    bool ds = false, dw = false;
    for (uint64_t v = tid; v <= nv; v += nt) ds |= ra[v] != rb[v];
    for (uint64_t e = tid; e < ne; e += nt) {
        ds |= ca[e] != cb[e];
        if (wa) dw |= wa[e] != wb[e];
    }
    if (__any_sync(kFullMask, ds) && (threadIdx.x & 31) == 0) atomicOr(diff, 1u);
    if (__any_sync(kFullMask, dw) && (threadIdx.x & 31) == 0) atomicOr(diff + 1, 1u);
}

// ------------------------------------------------------------------ edge list -> CSR

// Entry j of the build: input edge e = j >> rs, reversed when rs && (j & 1)
// (the reverse copies --d2ud inserts, samples/tools/gtools.cpp:224-238).
struct EdgeList {
    const uint32_t *src, *dst, *w;
    uint64_t m;
    uint32_t nv, rs;
    bool deself;
    __device__ __forceinline__ bool entry(uint64_t j, uint32_t &row, uint32_t &col) const {
        const uint64_t e = j >> rs;
        const bool rev = (j & rs) != 0;
        const uint32_t a = __ldg(src + e), b = __ldg(dst + e);
        row = rev ? b : a;
        col = rev ? a : b;
        return !(deself && a == b) && a < nv && b < nv;
    }
};

__global__ void count_entries_kernel(EdgeList el, uint32_t *deg, unsigned long long *first_bad) {
    const uint64_t n = el.m << el.rs;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t r, c;
        if (el.entry(j, r, c)) atomicAdd(deg + r, 1u);
        else if (r >= el.nv || c >= el.nv) atomicMin(first_bad, j >> el.rs);
    }
}

// Key of an entry: its position j (unique), above it the destination when
// rows are to be ordered or deduplicated by destination.
template <class K>
__global__ void scatter_entries_kernel(EdgeList el, uint32_t *cur, K *keys) {
    const uint64_t n = el.m << el.rs;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t r, c;
        if (!el.entry(j, r, c)) continue;
        const uint32_t p = atomicAdd(cur + r, 1u);
        if (sizeof(K) == 8) keys[p] = (K)(((uint64_t)c << 32) | j);
        else keys[p] = (K)j;
    }
}

// Deduplication over rows sorted by (destination, position): entry i survives
// when it opens its row or its destination differs from entry i-1's, i.e. the
// first key of each destination run (samples/tools/gtools.cpp:147-175 and the
// first-insert-wins map of 211-238).  Flat passes: a bitmap of row starts, a
// ballot word of survivors per 32 entries, a scan of the words' counts, then
// a coalesced compaction and the new row offsets.
__global__ void row_starts_kernel(const uint32_t *off, uint32_t nv, uint32_t *starts) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < nv; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t b = off[v];
        if (off[v + 1] > b) atomicOr(starts + (b >> 5), 1u << (b & 31));
    }
}

__global__ void unique_flags_kernel(const unsigned long long *keys, uint64_t n, const uint32_t *starts,
                                    uint32_t *words, uint32_t *counts) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = gw; w * 32 < n; w += nw) {
        const uint64_t i = w * 32 + lane;
        bool first = false;
        if (i < n) {
            first = ((starts[w] >> lane) & 1u) != 0;  // always set for entry 0
            if (!first) first = (keys[i] >> 32) != (keys[i - 1] >> 32);
        }
        const uint32_t word = __ballot_sync(kFullMask, first);
        if (lane == 0) {
            words[w] = word;
            counts[w] = __popc(word);
        }
    }
}

__global__ void unique_compact_kernel(const unsigned long long *keys, uint64_t n, const uint32_t *words,
                                      const uint32_t *wpos, uint32_t *kept) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t word = words[i >> 5], bit = (uint32_t)i & 31;
        if ((word >> bit) & 1u) kept[wpos[i >> 5] + __popc(word & ((1u << bit) - 1))] = (uint32_t)keys[i];
    }
}

// noff[v] = survivors before entry off[v]; words/wpos have one zero word past
// the data, so off[nv] == n reads the total.
__global__ void unique_offsets_kernel(const uint32_t *off, uint32_t nv, const uint32_t *words, const uint32_t *wpos,
                                      uint32_t *noff) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v <= nv; v += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = off[v], w = p >> 5;
        noff[v] = wpos[w] + __popc(words[w] & ((1u << (p & 31)) - 1));
    }
}

// Final columns and weights from the entries' positions.
template <class K>
__global__ void gather_entries_kernel(EdgeList el, const K *tags, uint64_t n, uint32_t *col, uint32_t *w) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)tags[i];
        const uint32_t e = j >> el.rs;
        const bool rev = (j & el.rs) != 0;
        col[i] = rev ? __ldg(el.src + e) : __ldg(el.dst + e);
        if (w) w[i] = __ldg(el.w + e);
    }
}

// Source of every CSR entry p: the row whose range holds p.
__device__ __forceinline__ uint32_t owner_row(const uint32_t *row, uint32_t nv, uint32_t p) {
    uint32_t lo = 0, hi = nv;  // largest u with row[u] <= p
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (__ldg(row + mid) <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void expand_rows_kernel(const uint32_t *row, uint32_t nv, uint64_t ne, uint32_t *src) {
    for (uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; p < ne; p += (uint64_t)gridDim.x * blockDim.x)
        src[p] = owner_row(row, nv, (uint32_t)p);
}

// A CSR built into temporaries of the call.
struct BuiltCsr {
    const uint32_t *row = nullptr, *col = nullptr, *w = nullptr;
    uint64_t ne = 0;
};

// Edge list -> CSR: count, scan, scatter, sort rows by (destination,
// position) when `sorted` or `dedup`, else by position alone; `dedup` keeps
// the first entry of every (source, destination).
sg_status build_rows(sg_ctx *ctx, Tmp &tmp, const EdgeList &el, bool sorted, bool dedup, BuiltCsr *out) {
    const cudaStream_t s = ctx->stream;
    const uint32_t nv = el.nv;
    const uint64_t n_in = el.m << el.rs;
    uint32_t *deg, *off;
    unsigned long long *bad;
    SG_TRY_CUDA(ctx, tmp.alloc(&deg, (uint64_t)nv + 1));
    SG_TRY_CUDA(ctx, tmp.alloc(&off, (uint64_t)nv + 1));
    SG_TRY_CUDA(ctx, tmp.alloc(&bad, 1));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(deg, 0, 4ull * (nv + 1), s));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(bad, 0xff, sizeof *bad, s));
    if (n_in) count_entries_kernel<<<grid_for(n_in, 256), 256, 0, s>>>(el, deg, bad);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    unsigned long long hbad = 0, n = 0;
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(&hbad, bad, sizeof hbad, cudaMemcpyDeviceToHost, s));
    sg_status st = exclusive_scan(ctx, tmp, deg, nv, off, &n);
    if (st != SG_OK) return st;
    if (hbad != ~0ull) return set_error(ctx, SG_ERR_INVALID_ARG, "edge %llu has an endpoint >= nv", hbad);
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(deg, off, 4ull * nv, cudaMemcpyDeviceToDevice, s));  // scatter cursors

    const uint32_t *row = off;
    uint64_t ne = n;
    const void *tags = nullptr;
    bool tags64 = false;
    if (sorted || dedup) {
        unsigned long long *keys;
        SG_TRY_CUDA(ctx, tmp.alloc(&keys, n));
        if (n) scatter_entries_kernel<unsigned long long><<<grid_for(n_in, 256), 256, 0, s>>>(el, deg, keys);
        SG_TRY_CUDA(ctx, cudaGetLastError());
        if ((st = sort_rows<unsigned long long>(ctx, off, nv, n, keys)) != SG_OK) return st;
        if (dedup) {
            const uint64_t nwords = (n + 31) / 32 + 1;  // one zero word past the data
            uint32_t *starts, *words, *wcount, *wpos, *noff, *kept;
            SG_TRY_CUDA(ctx, tmp.alloc(&starts, nwords));
            SG_TRY_CUDA(ctx, tmp.alloc(&words, nwords));
            SG_TRY_CUDA(ctx, tmp.alloc(&wcount, nwords));
            SG_TRY_CUDA(ctx, tmp.alloc(&wpos, nwords + 1));
            SG_TRY_CUDA(ctx, tmp.alloc(&noff, (uint64_t)nv + 1));
            SG_TRY_CUDA(ctx, cudaMemsetAsync(starts, 0, 4 * nwords, s));
            SG_TRY_CUDA(ctx, cudaMemsetAsync(words, 0, 4 * nwords, s));
            SG_TRY_CUDA(ctx, cudaMemsetAsync(wcount, 0, 4 * nwords, s));
            row_starts_kernel<<<grid_for(nv, 256), 256, 0, s>>>(off, nv, starts);
            if (n) unique_flags_kernel<<<grid_for(n, 256), 256, 0, s>>>(keys, n, starts, words, wcount);
            SG_TRY_CUDA(ctx, cudaGetLastError());
            unsigned long long nk = 0;
            if ((st = exclusive_scan(ctx, tmp, wcount, nwords, wpos, &nk)) != SG_OK) return st;
            SG_TRY_CUDA(ctx, tmp.alloc(&kept, nk));
            if (n) unique_compact_kernel<<<grid_for(n, 256), 256, 0, s>>>(keys, n, words, wpos, kept);
            unique_offsets_kernel<<<grid_for((uint64_t)nv + 1, 256), 256, 0, s>>>(off, nv, words, wpos, noff);
            SG_TRY_CUDA(ctx, cudaGetLastError());
            // without row ordering the survivors go back to input order
            if (!sorted && (st = sort_rows<uint32_t>(ctx, noff, nv, nk, kept)) != SG_OK) return st;
            row = noff;
            ne = nk;
            tags = kept;
        } else {
            tags = keys;
            tags64 = true;
        }
    } else {
        uint32_t *keys;
        SG_TRY_CUDA(ctx, tmp.alloc(&keys, n));
        if (n) scatter_entries_kernel<uint32_t><<<grid_for(n_in, 256), 256, 0, s>>>(el, deg, keys);
        SG_TRY_CUDA(ctx, cudaGetLastError());
        if ((st = sort_rows<uint32_t>(ctx, off, nv, n, keys)) != SG_OK) return st;
        tags = keys;
    }
    uint32_t *col, *w = nullptr;
    SG_TRY_CUDA(ctx, tmp.alloc(&col, ne));
    if (el.w) SG_TRY_CUDA(ctx, tmp.alloc(&w, ne));
    if (ne) {
        if (tags64)
            gather_entries_kernel<unsigned long long><<<grid_for(ne, 256), 256, 0, s>>>(el, (const unsigned long long *)tags, ne, col, w);
        else
            gather_entries_kernel<uint32_t><<<grid_for(ne, 256), 256, 0, s>>>(el, (const uint32_t *)tags, ne, col, w);
    }
    SG_TRY_CUDA(ctx, cudaGetLastError());
    out->row = row;
    out->col = col;
    out->w = w;
    out->ne = ne;
    return SG_OK;
}

}  // namespace gbuild

// CSR (device arrays) -> CSC into crow (nv+1), ccol (ne) and cw (ne, when w).
sg_status device_transpose(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *row, const uint32_t *col,
                           const uint32_t *w, uint32_t *crow, uint32_t *ccol, uint32_t *cw) {
    using namespace gbuild;
    const cudaStream_t s = ctx->stream;
    Tmp tmp(ctx, "tr");
    uint32_t *cnt;
    SG_TRY_CUDA(ctx, tmp.alloc(&cnt, (uint64_t)nv + 1));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(cnt, 0, 4ull * (nv + 1), s));
    count_by_col_kernel<<<grid_for(ne, 256), 256, 0, s>>>(col, ne, cnt);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    unsigned long long total = 0;
    sg_status st = exclusive_scan(ctx, tmp, cnt, nv, crow, &total);
    if (st != SG_OK) return st;
    if (total != ne) return set_error(ctx, SG_ERR_CUDA, "transpose counted %llu of %llu edges", total, (unsigned long long)ne);
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(cnt, crow, 4ull * nv, cudaMemcpyDeviceToDevice, s));
    scatter_by_col_kernel<<<grid_for(ne, 256), 256, 0, s>>>(col, ne, cnt, ccol);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    st = sort_rows<uint32_t>(ctx, crow, nv, ne, ccol);
    if (st != SG_OK) return st;
    csc_finish_kernel<<<grid_for(ne, 256), 256, 0, s>>>(row, nv, w, ne, ccol, cw);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    return SG_OK;
}

// Structure and weights of two device CSRs of the same size differ?
sg_status device_compare_csr(sg_ctx *ctx, uint32_t nv, uint64_t ne, const uint32_t *ra, const uint32_t *ca,
                             const uint32_t *wa, const uint32_t *rb, const uint32_t *cb, const uint32_t *wb,
                             bool *structure_differs, bool *weights_differ) {
    using namespace gbuild;
    const cudaStream_t s = ctx->stream;
    Tmp tmp(ctx, "cmp");
    uint32_t *diff, hd[2];
    SG_TRY_CUDA(ctx, tmp.alloc(&diff, 2));
    SG_TRY_CUDA(ctx, cudaMemsetAsync(diff, 0, 8, s));
    compare_csr_kernel<<<grid_for(std::max<uint64_t>(ne, nv), 256), 256, 0, s>>>(ra, rb, nv, ca, cb, wa, wb, ne, diff);
    SG_TRY_CUDA(ctx, cudaGetLastError());
    SG_TRY_CUDA(ctx, cudaMemcpyAsync(hd, diff, sizeof hd, cudaMemcpyDeviceToHost, s));
    SG_TRY_CUDA(ctx, cudaStreamSynchronize(s));
    *structure_differs = hd[0] != 0;
    *weights_differ = hd[1] != 0;
    return SG_OK;
}

// In-edge view of a symmetric weighted graph.  A symmetric graph's CSC
// aliases its CSR (csr_graph.h:405-410); with weights that alias is right
// only when the transpose has the same structure and w(u->v) == w(v->u) edge
// by edge.  An identical structure keeps the alias and gets its own CSC weight
// array when the weights differ; any other structure gets a full CSC.
sg_status symmetric_weighted_csc(sg_ctx *ctx, sg_graph *g) {
    using namespace gbuild;
    const uint32_t nv = g->nv;
    const uint64_t ne = g->ne;
    Tmp tmp(ctx, "sym");
    uint32_t *trow, *tcol, *tw;
    SG_TRY_CUDA(ctx, tmp.alloc(&trow, (uint64_t)nv + 1));
    SG_TRY_CUDA(ctx, tmp.alloc(&tcol, ne));
    SG_TRY_CUDA(ctx, tmp.alloc(&tw, ne));
    sg_status st = device_transpose(ctx, nv, ne, g->row, g->col, g->w, trow, tcol, tw);
    if (st != SG_OK) return st;
    bool sd = false, wd = false;
    st = device_compare_csr(ctx, nv, ne, g->row, g->col, g->w, trow, tcol, tw, &sd, &wd);
    if (st != SG_OK || (!sd && !wd)) return st;
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_row = al(4ull * (nv + 1)), b_col = al(4ull * std::max<uint64_t>(ne, 1));
    const size_t total = b_row + 2 * b_col + (sd ? b_row + 2 * b_col : b_col);
    void *arena = nullptr;
    SG_TRY_CUDA(ctx, cudaMalloc(&arena, total));
    char *p = (char *)arena;
    auto carve = [&](size_t bytes) {
        uint32_t *q = (uint32_t *)p;
        p += bytes;
        return q;
    };
    uint32_t *row = carve(b_row), *col = carve(b_col), *w = carve(b_col);
    uint32_t *crow = row, *ccol = col, *cw;
    if (sd) {
        crow = carve(b_row);
        ccol = carve(b_col);
    }
    cw = carve(b_col);
    const cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(row, g->row, 4ull * (nv + 1), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && ne) e = cudaMemcpyAsync(col, g->col, 4ull * ne, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && ne) e = cudaMemcpyAsync(w, g->w, 4ull * ne, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && sd) e = cudaMemcpyAsync(crow, trow, 4ull * (nv + 1), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && sd && ne) e = cudaMemcpyAsync(ccol, tcol, 4ull * ne, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && ne) e = cudaMemcpyAsync(cw, tw, 4ull * ne, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(arena);
        return cuda_status(ctx, e, "graph relayout");
    }
    cudaFree(g->arena);
    g->arena = arena;
    g->arena_bytes = total;
    g->row = row;
    g->col = col;
    g->w = w;
    g->crow = crow;
    g->ccol = ccol;
    g->cw = cw;
    return SG_OK;
}

}  // namespace sgb

extern "C" {

sg_status sg_graph_build(sg_ctx *ctx, uint32_t nv, uint64_t m, const uint32_t *src, const uint32_t *dst,
                         const uint32_t *weights, uint32_t build_flags, uint32_t graph_flags, sg_graph **out) {
    using namespace sgb;
    using namespace sgb::gbuild;
    if (!ctx || !out || nv == 0 || (m && (!src || !dst)) || nv == 0xffffffffu) return SG_ERR_INVALID_ARG;
    if (build_flags & ~(SG_BUILD_DESELF_CYCLE | SG_BUILD_DEDUPLICATE | SG_BUILD_D2UD | SG_BUILD_SORT_ROWS))
        return set_error(ctx, SG_ERR_INVALID_ARG, "unknown build flags 0x%x", build_flags);
    *out = nullptr;
    DeviceGuard dg(ctx->device);
    const bool d2ud = build_flags & SG_BUILD_D2UD;
    const bool dedup = d2ud || (build_flags & SG_BUILD_DEDUPLICATE);
    const bool sorted = d2ud || (build_flags & SG_BUILD_SORT_ROWS);
    if (m > kMaxEntries) return set_error(ctx, SG_ERR_INVALID_ARG, "%llu edges exceed the uint32 entry range", (unsigned long long)m);
    if (d2ud) graph_flags |= SG_GRAPH_SYMMETRIC;
    const cudaStream_t s = ctx->stream;
    Tmp tmp(ctx, "in");

    // inputs on the device
    EdgeList el{src, dst, weights, m, nv, 0u, (build_flags & SG_BUILD_DESELF_CYCLE) != 0};
    auto on_device = [&](const uint32_t *p, const uint32_t **dp) -> sg_status {
        if (!p || is_device_ptr(p, ctx->device)) {
            *dp = p;
            return SG_OK;
        }
        uint32_t *q;
        SG_TRY_CUDA(ctx, tmp.alloc(&q, m));
        SG_TRY_CUDA(ctx, cudaMemcpyAsync(q, p, 4 * m, cudaMemcpyDefault, s));
        *dp = q;
        return SG_OK;
    };
    sg_status st;
    if (m) {
        if ((st = on_device(src, &el.src)) != SG_OK) return st;
        if ((st = on_device(dst, &el.dst)) != SG_OK) return st;
        if ((st = on_device(weights, &el.w)) != SG_OK) return st;
    }
    // The converter works on a CSR whose rows hold each source's edges in
    // input order; --d2ud then inserts edges in that CSR order (first insert
    // wins), so it runs as a second pass over the CSR built first.
    BuiltCsr a;
    if ((st = build_rows(ctx, tmp, el, sorted && !d2ud, dedup && !d2ud, &a)) != SG_OK) return st;
    if (d2ud) {
        if (2 * a.ne > kMaxEntries)
            return set_error(ctx, SG_ERR_INVALID_ARG, "%llu edges doubled by d2ud exceed the uint32 entry range",
                             (unsigned long long)a.ne);
        uint32_t *src2;
        SG_TRY_CUDA(ctx, tmp.alloc(&src2, a.ne));
        if (a.ne) expand_rows_kernel<<<grid_for(a.ne, 256), 256, 0, s>>>(a.row, nv, a.ne, src2);
        SG_TRY_CUDA(ctx, cudaGetLastError());
        const EdgeList el2{src2, a.col, a.w, a.ne, nv, 1u, false};
        if ((st = build_rows(ctx, tmp, el2, true, true, &a)) != SG_OK) return st;
    }
    return create_graph(ctx, nv, a.ne, a.row, a.col, a.w, graph_flags, out);
}

}  // extern "C"
