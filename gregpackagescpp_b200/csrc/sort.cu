// Device scan and a stable LSD radix sort of 64-bit keys with 32-bit values (8-bit digits).
// Used for the Morton order of the octree build (greg8tree.hpp leaf order = ascending code) and
// for the spatial reordering of the direct-sum bodies.
#include <cuda_runtime.h>

#include <atomic>

#include "gtd_internal.cuh"
#include "gtd_sort.cuh"

namespace gtd {

constexpr int kSortThreads = 256;
constexpr int kHalfItems = 8;                        // keys per thread per chunk
constexpr int kHalf = kSortThreads * kHalfItems;     // keys per chunk (a block takes a run of chunks)
constexpr int kScatterBlocksPerSm = 4;               // the scatter's launch bound (at most 64 registers)
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

// ---- exclusive scan of uint32 (arbitrary length, three phases) ---------------------------------
__global__ void scan_tiles_kernel(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *tile_sums) {
    __shared__ uint32_t warp_tot[kScanThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems], run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        v[k] = i < n ? in[i] : 0u;
        const uint32_t t = v[k];
        v[k] = run;
        run += t;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = wi - w;
        if (lane == kScanThreads / 32 - 1 && tile_sums) tile_sums[blockIdx.x] = wi;
    }
    __syncthreads();
    const uint32_t off = warp_tot[warp] + incl - run;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (i < n) out[i] = v[k] + off;
    }
}

__global__ void scan_add_kernel(uint32_t *out, int64_t n, const uint32_t *tile_offsets) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += tile_offsets[i / kScanTile];
}

size_t scan_scratch_words(int64_t n) {
    size_t words = 0;
    int64_t m = n;
    while (m > kScanTile) {
        m = (m + kScanTile - 1) / kScanTile;
        words += (size_t)m;
    }
    return words + 1;
}

// Exclusive scan in -> out (may alias).  scratch: scan_scratch_words(n) words.
int exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *scratch, cudaStream_t s,
                       uint64_t *launches) {
    if (n <= 0) return GTD_OK;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles == 1) {
        scan_tiles_kernel<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
        GTD_CHECK_LAUNCH();
        if (launches) *launches += 1;
        return GTD_OK;
    }
    uint32_t *sums = scratch;
    scan_tiles_kernel<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums);
    GTD_CHECK_LAUNCH();
    int rc = exclusive_scan_u32(sums, sums, tiles, scratch + tiles, s, launches);
    if (rc) return rc;
    scan_add_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(out, n, sums);
    GTD_CHECK_LAUNCH();
    if (launches) *launches += 2;
    return GTD_OK;
}

// ---- radix sort ----------------------------------------------------------------------------
// Block b of a pass owns the keys [b * per_block, (b + 1) * per_block), per_block a whole number of
// kHalf-key chunks: the grid is one wave of the scatter kernel, whatever n is (radix_grid).
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const unsigned long long *keys, int64_t n,
                                                                  int shift, uint32_t *hist, int blocks,
                                                                  int64_t per_block) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * per_block;
    const int64_t end = min(base + per_block, n);
    for (int64_t i = base + threadIdx.x; i < end; i += kSortThreads) atomicAdd(&h[(keys[i] >> shift) & 0xffu], 1u);
    __syncthreads();
    hist[(size_t)threadIdx.x * blocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter.  A block takes its keys in chunks of kHalf.  In a chunk, warp w owns the
// contiguous keys w*256 .. w*256+255 (eight rounds of 32, in index order) and ranks them stably
// inside its own digit counters (match_any per round, warp-synchronous: no block barrier); one block
// scan over the 256 digits then turns the per-warp counts into offsets, the keys are placed
// digit-sorted in shared memory and written out in that order: keys of one digit go to consecutive
// addresses, so the stores fill whole sectors instead of one 8-byte store per key.  Seven block
// barriers per chunk (the earlier block-wide ranking rounds took 34).
__global__ void __launch_bounds__(kSortThreads, kScatterBlocksPerSm) radix_scatter_kernel(
    const unsigned long long *keys_in, const int32_t *vals_in, unsigned long long *keys_out, int32_t *vals_out,
    int64_t n, int shift, const uint32_t *offsets, int blocks, int64_t per_block) {
    constexpr int kWarps = kSortThreads / 32;
    static_assert(kHalf == kWarps * 32 * kHalfItems, "a warp owns kHalfItems rounds of 32 keys");
    __shared__ unsigned long long sk[kHalf];
    __shared__ int32_t sv[kHalf];
    __shared__ uint32_t wcnt[kWarps][256];  // per-warp digit counts, then per-warp digit offsets
    __shared__ uint32_t pre[256], run_global[256], wsum[kWarps];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const unsigned lt = (1u << lane) - 1u;
    run_global[t] = offsets[(size_t)t * blocks + blockIdx.x];
    const int64_t base = (int64_t)blockIdx.x * per_block;
    const int64_t end = min(base + per_block, n);
    for (int64_t hbase = base; hbase < end; hbase += kHalf) {
        unsigned long long key[kHalfItems];
        int32_t val[kHalfItems];
        uint32_t dig[kHalfItems], wr[kHalfItems];
#pragma unroll
        for (int w = 0; w < kWarps; ++w) wcnt[w][t] = 0;
#pragma unroll
        for (int k = 0; k < kHalfItems; ++k) {
            const int64_t i = hbase + (int64_t)warp * (32 * kHalfItems) + k * 32 + lane;
            key[k] = 0;
            val[k] = 0;
            dig[k] = 256;  // absent keys get a digit no key has
            if (i < end) {
                key[k] = keys_in[i];
                val[k] = vals_in[i];
                dig[k] = (uint32_t)((key[k] >> shift) & 0xffu);
            }
        }
        __syncthreads();
        // stable rank inside the warp: rounds in index order, lanes in index order within a round
#pragma unroll
        for (int k = 0; k < kHalfItems; ++k) {
            const uint32_t d = dig[k];
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const unsigned rank = __popc(peers & lt);
            const uint32_t before = d < 256 ? wcnt[warp][d] : 0u;
            __syncwarp();
            if (d < 256 && rank == 0) wcnt[warp][d] = before + __popc(peers);
            __syncwarp();
            wr[k] = before + rank;
        }
        __syncthreads();
        // digit totals of the half and their exclusive scan, one digit per thread
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) c += wcnt[w][t];
        uint32_t incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t wofs = 0;
        for (int w = 0; w < warp; ++w) wofs += wsum[w];
        const uint32_t start = wofs + incl - c;
        pre[t] = start;
        // per-warp offsets of digit t inside the half: warps in order
        uint32_t run = start;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t cw = wcnt[w][t];
            wcnt[w][t] = run;
            run += cw;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kHalfItems; ++k) {
            const uint32_t d = dig[k];
            if (d < 256) {
                const uint32_t pos = wcnt[warp][d] + wr[k];
                if (pos < (uint32_t)kHalf) {
                    sk[pos] = key[k];
                    sv[pos] = val[k];
                }
            }
        }
        __syncthreads();
        const int64_t rem = end - hbase;
        const int hcount = rem < kHalf ? (int)rem : kHalf;
#pragma unroll
        for (int k = 0; k < kHalfItems; ++k) {
            const int i = k * kSortThreads + t;
            if (i < hcount) {
                const unsigned long long kk = sk[i];
                const uint32_t d = (uint32_t)((kk >> shift) & 0xffu);
                const uint32_t g = run_global[d] + (uint32_t)i - pre[d];
                if ((int64_t)g < n) {
                    keys_out[g] = kk;
                    vals_out[g] = sv[i];
                }
            }
        }
        __syncthreads();
        run_global[t] += c;
        __syncthreads();
    }
}

// The scatter's resident blocks per SM on the current device (its launch bound or less), looked up
// once per device; handles on different host threads may sort at the same time.
static int scatter_blocks_per_sm() {
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
    std::atomic<int> *c = dev < 64 ? &cached[dev] : nullptr;
    if (c) {
        const int v = c->load(std::memory_order_relaxed);
        if (v > 0) return v;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, radix_scatter_kernel, kSortThreads, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    if (c) c->store(per_sm, std::memory_order_relaxed);
    return per_sm;
}

// Grid of a pass: blocks of a whole number of chunks each, as few chunks per block as one wave of
// the scatter kernel allows (a second, partial wave would cost as much as the first).
static void radix_grid(int64_t n, int *blocks, int64_t *per_block) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 148;
    const int64_t slots = (int64_t)sms * scatter_blocks_per_sm();
    const int64_t chunks = (n + kHalf - 1) / kHalf;
    const int64_t cpb = (chunks + slots - 1) / slots;
    *per_block = cpb * kHalf;
    *blocks = (int)((chunks + cpb - 1) / cpb);
}

// Sized for one block per chunk, the most any device's grid takes.
size_t radix_scratch_words(int64_t n) {
    const int64_t blocks = (n + kHalf - 1) / kHalf;
    const int64_t h = 256 * blocks;
    return (size_t)h + scan_scratch_words(h);
}

// Sorts (keys, vals) by the bits [0, bits) of the keys, stably.  Uses (keys_alt, vals_alt) as the
// ping-pong buffers; the result lands back in (keys, vals).
int radix_sort_u64(unsigned long long *keys, int32_t *vals, unsigned long long *keys_alt, int32_t *vals_alt,
                   int64_t n, int bits, uint32_t *scratch, cudaStream_t s, uint64_t *launches) {
    if (n <= 1) return GTD_OK;
    int blocks = 1;
    int64_t per_block = kHalf;
    radix_grid(n, &blocks, &per_block);
    uint32_t *hist = scratch;
    uint32_t *scan_scratch = scratch + (size_t)256 * blocks;
    unsigned long long *ka = keys, *kb = keys_alt;
    int32_t *va = vals, *vb = vals_alt;
    int passes = 0;
    for (int shift = 0; shift < bits; shift += 8, ++passes) {
        radix_hist_kernel<<<blocks, kSortThreads, 0, s>>>(ka, n, shift, hist, blocks, per_block);
        GTD_CHECK_LAUNCH();
        int rc = exclusive_scan_u32(hist, hist, (int64_t)256 * blocks, scan_scratch, s, launches);
        if (rc) return rc;
        radix_scatter_kernel<<<blocks, kSortThreads, 0, s>>>(ka, va, kb, vb, n, shift, hist, blocks, per_block);
        GTD_CHECK_LAUNCH();
        if (launches) *launches += 2;
        unsigned long long *tk = ka; ka = kb; kb = tk;
        int32_t *tv = va; va = vb; vb = tv;
    }
    if (ka != keys) {
        GTD_CUDA(cudaMemcpyAsync(keys, ka, sizeof(unsigned long long) * (size_t)n, cudaMemcpyDeviceToDevice, s));
        GTD_CUDA(cudaMemcpyAsync(vals, va, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, s));
    }
    return GTD_OK;
}

}  // namespace gtd
