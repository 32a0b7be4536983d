// (b) Tile|depth ordering: stable LSD radix sort, exclusive scan, depth-ordered
// record emission and per-tile ranges.
//
// The reference sorts one (tile << 32 | depth bits) 64-bit key per record with
// a stable radix sort over 32 + ceil(log2 T) bits (renderer.cu:223-271, 541-563).
// Here the same order - tile ascending, then depth bits ascending, then Gaussian
// id ascending - is produced with far less traffic:
//   1. a stable 32-bit radix sort of the N per-Gaussian depth keys (ids as values),
//   2. records emitted in that depth order (exclusive scan of tile counts),
//   3. a stable radix sort of the R records on the ceil(log2 T) tile bits only.
// Stability of step 3 keeps depth (then id) order inside every tile, so the
// resulting per-tile lists equal the reference's bit for bit.
//
// Every kernel reads its element count from device memory when one is given, so
// the whole chain runs without a host round trip and can be captured in a graph.
#include "common.cuh"
#include "kernels.h"

#include <mutex>

namespace gsn {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
// 12 keys per thread measured fastest (8: tile sort 0.139 ms, 12: 0.128 ms, 16:
// 0.136 ms at 7.2M records): longer scatter runs against fewer CTAs per SM
constexpr int kSortItems = 12;                      // per thread
constexpr int kSortChunk = kSortThreads * kSortItems;  // 3072 keys per block
constexpr int kBins = 256;
// Each pass's digit totals are kept as kTotalCopies partial copies, one 1 KB row
// apart, and a block adds into copy blockIdx % kTotalCopies: the thousands of
// blocks of a pass then spread their global atomics over as many L2 lines
// instead of queueing on the four lines of a single 256-word row.
constexpr int kTotalCopies = 16;
// per-block counts per thread in radix_scan (12, one round for the 2,367 blocks of
// 7.2M records, measured slower: tile sort 0.113 -> 0.115 ms)
constexpr int kScanPer = 4;
constexpr uint32_t kSortSentinel = 0xFFFFFFFFu;  // the key a dropping sort leaves out

// Device-resident counts are clamped to the host-side capacity the grid was sized
// for, so an overflowing count can never drive an access past the buffers.
__device__ __forceinline__ int load_count(const int* dev, int host) { return dev ? min(*dev, host) : host; }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Per-block digit histogram of one digit of at most 8 bits (digits <= mask).
template <bool kDrop>
__global__ void __launch_bounds__(kSortThreads) radix_upsweep(const uint32_t* __restrict__ keys,
                                                              const int* n_dev, int n_host, int bit, uint32_t mask,
                                                              uint32_t* __restrict__ block_hist,
                                                              size_t hist_stride,
                                                              uint32_t* __restrict__ digit_total) {
    pdl_begin();
    __shared__ uint32_t hist[kSortWarps][kBins];
    const int n = load_count(n_dev, n_host);
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kSortChunk;
    if (start >= n) return;
    const int64_t end = min(static_cast<int64_t>(n), start + kSortChunk);
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kBins; i += kSortThreads) (&hist[0][0])[i] = 0;
    __syncthreads();
    // the chunk's loads first, then the shared-memory counts
    uint32_t key[kSortItems];
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t idx = start + k * kSortThreads + threadIdx.x;
        key[k] = idx < end ? __ldg(keys + idx) : kSortSentinel;
    }
#pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t idx = start + k * kSortThreads + threadIdx.x;
        if (idx < end && (!kDrop || key[k] != kSortSentinel)) atomicAdd(&hist[warp][(key[k] >> bit) & mask], 1u);
    }
    __syncthreads();
    const int d = threadIdx.x;
    if (d > static_cast<int>(mask)) return;  // rows of digits this pass cannot have stay unwritten
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) total += hist[w][d];
    block_hist[d * hist_stride + blockIdx.x] = total;
    if (total) atomicAdd(digit_total + (blockIdx.x % kTotalCopies) * kBins + d, total);
}

// A digit's total: the sum of its partial copies.
__device__ __forceinline__ uint32_t digit_sum(const uint32_t* __restrict__ digit_total, int d) {
    uint32_t v = 0;
#pragma unroll
    for (int c = 0; c < kTotalCopies; ++c) v += digit_total[c * kBins + d];
    return v;
}

// One block per digit: exclusive scan of that digit's per-block counts, offset by
// the number of keys with a smaller digit.
__global__ void __launch_bounds__(kSortThreads) radix_scan(const int* n_dev, int n_host,
                                                           uint32_t* __restrict__ block_hist,
                                                           size_t hist_stride,
                                                           const uint32_t* __restrict__ digit_total) {
    pdl_begin();
    __shared__ uint32_t warp_sums[kSortWarps];
    __shared__ uint32_t carry;
    const int n = load_count(n_dev, n_host);
    const int blocks = ceil_div(n, kSortChunk);
    const int d = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // base = sum of totals of smaller digits
    uint32_t v = threadIdx.x < d ? digit_sum(digit_total, threadIdx.x) : 0u;
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) warp_sums[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kSortWarps; ++w) s += warp_sums[w];
        carry = s;
    }
    __syncthreads();
    uint32_t* row = block_hist + d * hist_stride;
    // kScanPer consecutive counts per thread: a quarter of the rounds (and of
    // their barriers) of one count per thread
    for (int base = 0; base < blocks; base += kSortThreads * kScanPer) {
        const int i0 = base + threadIdx.x * kScanPer;
        uint32_t x[kScanPer];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            x[k] = i0 + k < blocks ? row[i0 + k] : 0u;
            sum += x[k];
        }
        // inclusive warp scan of the thread sums
        uint32_t inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        __syncthreads();
        if (lane == 31) warp_sums[warp] = inc;
        __syncthreads();
        uint32_t warp_prefix = 0, chunk_total = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t s = warp_sums[w];
            if (w < warp) warp_prefix += s;
            chunk_total += s;
        }
        const uint32_t c = carry;
        uint32_t run = c + warp_prefix + inc - sum;
#pragma unroll
        for (int k = 0; k < kScanPer; ++k) {
            if (i0 + k < blocks) row[i0 + k] = run;
            run += x[k];
        }
        __syncthreads();
        if (threadIdx.x == 0) carry = c + chunk_total;
    }
}

// Stable scatter. Warp w owns the w-th 384-key slice of the block's chunk and
// walks it in 32-key steps; eight ballots (one per digit bit) find the lanes with
// an equal digit inside a step, and
// warp-private counters carry the rank across steps, which keeps the original
// order among equal digits. The ranked keys are first placed digit-sorted in
// shared memory and then written out linearly, so each warp store covers a run
// of consecutive addresses of one digit bucket instead of 32 scattered words.
template <bool kIdentityValues, bool kDrop>
__global__ void __launch_bounds__(kSortThreads) radix_downsweep(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ values_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ values_out, const int* n_dev, int n_host,
    int bit, uint32_t mask, int digit_bits, const uint32_t* __restrict__ block_hist, size_t hist_stride) {
    pdl_begin();
    __shared__ uint32_t counts[kSortWarps][kBins];
    __shared__ uint32_t global_base[kBins];
    __shared__ uint32_t local_base[kBins];
    __shared__ uint32_t s_keys[kSortChunk];
    __shared__ uint32_t s_vals[kSortChunk];
    const int n = load_count(n_dev, n_host);
    const int64_t start = static_cast<int64_t>(blockIdx.x) * kSortChunk;
    if (start >= n) return;
    const int64_t end = min(static_cast<int64_t>(n), start + kSortChunk);
    __shared__ int s_total;  // keys of this chunk that are written (all but dropped sentinels)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * kBins; i += kSortThreads) (&counts[0][0])[i] = 0;
    // only the rows of digits <= mask were written (and scanned) for this pass
    global_base[threadIdx.x] =
        threadIdx.x <= mask ? block_hist[threadIdx.x * hist_stride + blockIdx.x] : 0u;
    __syncthreads();

    const uint32_t lt = lanemask_lt();
    const int64_t slice = start + static_cast<int64_t>(warp) * (kSortItems * 32);
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
    // all of the slice's loads first, so they are in flight together (the
    // warp-synchronous ranking below would otherwise wait for each step's pair)
#pragma unroll
    for (int s = 0; s < kSortItems; ++s) {
        const int64_t idx = slice + s * 32 + lane;
        const bool valid = idx < end;
        key[s] = valid ? keys_in[idx] : 0u;
        if (kIdentityValues) val[s] = static_cast<uint32_t>(idx);
        else val[s] = valid ? values_in[idx] : 0u;
    }
#pragma unroll
    for (int s = 0; s < kSortItems; ++s) {
        bool valid = slice + s * 32 + lane < end;
        if (kDrop) valid = valid && key[s] != kSortSentinel;
        uint32_t digit = valid ? ((key[s] >> bit) & mask) : 0u;
        // lanes holding the same digit: intersect the per-bit ballots of the
        // pass's digit bits
        uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            if (b >= digit_bits) break;
            uint32_t bal = __ballot_sync(0xffffffffu, (digit >> b) & 1u);
            peers &= ((digit >> b) & 1u) ? bal : ~bal;
        }
        uint32_t before = 0;
        if (valid) before = counts[warp][digit];
        __syncwarp();
        rank[s] = valid ? before + __popc(peers & lt) : 0xFFFFFFFFu;
        if (valid && (peers & lt) == 0) counts[warp][digit] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {   // exclusive prefix over warps per digit, then over digits for the block
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            uint32_t c = counts[w][d];
            counts[w][d] = run;
            run += c;
        }
        // block-wide exclusive scan of the per-digit totals
        uint32_t inc = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        __shared__ uint32_t warp_tot[kSortWarps];
        if (lane == 31) warp_tot[warp] = inc;
        __syncthreads();
        uint32_t prefix = 0, all = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            if (w < warp) prefix += warp_tot[w];
            all += warp_tot[w];
        }
        local_base[d] = prefix + inc - run;
        if (kDrop && d == 0) s_total = static_cast<int>(all);
    }
    __syncthreads();
    const int total = kDrop ? s_total : static_cast<int>(end - start);
#pragma unroll
    for (int s = 0; s < kSortItems; ++s) {
        if (rank[s] == 0xFFFFFFFFu) continue;
        uint32_t digit = (key[s] >> bit) & mask;
        uint32_t pos = local_base[digit] + counts[warp][digit] + rank[s];
        s_keys[pos] = key[s];
        s_vals[pos] = val[s];
    }
    __syncthreads();
    for (int j = threadIdx.x; j < total; j += kSortThreads) {
        uint32_t k = s_keys[j];
        uint32_t digit = (k >> bit) & mask;
        uint32_t pos = global_base[digit] + (j - local_base[digit]);
        keys_out[pos] = k;
        values_out[pos] = s_vals[j];
    }
}

// Keys kept by a dropping first pass: the sum of its digit totals.
__global__ void radix_kept(const uint32_t* __restrict__ digit_total, int* __restrict__ kept) {
    pdl_begin();
    __shared__ uint32_t part[kSortWarps];
    uint32_t v = digit_sum(digit_total, threadIdx.x);
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kSortWarps; ++w) s += part[w];
        *kept = static_cast<int>(s);
    }
}

// ---------------------------------------------------------------- scan
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int x, int* warp_sums, int* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sums[warp] = inc;
    __syncthreads();
    int prefix = 0, sum = 0;
#pragma unroll
    for (int w = 0; w < kScanThreads / 32; ++w) {
        int s = warp_sums[w];
        if (w < warp) prefix += s;
        sum += s;
    }
    __syncthreads();
    *total = sum;
    return prefix + inc - x;
}

// Single-pass exclusive scan with decoupled look-back (Merrill and Garland
// 2016). A CTA takes the next chunk index from a ticket counter (so every chunk
// it waits on belongs to a CTA that has already started), scans its chunk in
// shared memory, publishes the chunk total (aggregate; chunk 0 publishes its
// inclusive prefix at once) and lets warp 0 read the 32 preceding chunks' status
// words at a time: it adds aggregates up to the nearest inclusive prefix and
// publishes its own. Status words hold the flag in the top two bits and the
// value below. A word that stays unpublished for kScanPolls polls sets *error
// and ends the walk; offsets then come out too small but never negative, and
// every write stays inside the n + 1 outputs.
constexpr uint64_t kScanAggregate = 1ull << 62;
constexpr uint64_t kScanInclusive = 2ull << 62;
constexpr uint64_t kScanValue = (1ull << 62) - 1;
constexpr int kScanPolls = 1 << 20;

__device__ __forceinline__ void store_scan_status(unsigned long long* address, unsigned long long value) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(address), "l"(value) : "memory");
}

__device__ __forceinline__ unsigned long long load_scan_status(const unsigned long long* address) {
    unsigned long long value;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(value) : "l"(address) : "memory");
    return value;
}

__device__ __forceinline__ long long warp_sum64(long long v) {
#pragma unroll
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void __launch_bounds__(kScanThreads) scan_onepass(const int* in, const uint32_t* __restrict__ gather,
                                                             int n, const int* __restrict__ valid_dev, int* out,
                                                             unsigned long long* __restrict__ status,
                                                             int* __restrict__ ticket, int* __restrict__ error) {
    pdl_begin();
    __shared__ int warp_sums[kScanThreads / 32];
    __shared__ int tile[kScanChunk];
    __shared__ int s_chunk;
    __shared__ long long s_excl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_chunk = atomicAdd(ticket, 1);
    __syncthreads();
    const int chunk = s_chunk;
    const int64_t start = static_cast<int64_t>(chunk) * kScanChunk;
    const int valid = valid_dev ? min(*valid_dev, n) : n;
    // striped coalesced load -> blocked per-thread sequences via shared memory;
    // entries from `valid` on count as zero
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const int64_t i = start + j;
        tile[j] = i < valid ? (gather ? in[gather[i]] : in[i]) : 0;
    }
    __syncthreads();
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = tile[threadIdx.x * kScanItems + k];
        sum += v[k];
    }
    int total;
    int run = block_exclusive_scan(sum, warp_sums, &total);
    if (threadIdx.x == 0) {
        store_scan_status(status + chunk, (chunk == 0 ? kScanInclusive : kScanAggregate) |
                                              static_cast<unsigned long long>(total));
        if (chunk == 0) s_excl = 0;
    }
    if (chunk > 0 && warp == 0) {
        long long excl = 0;
        int c = chunk - 1;  // the nearest chunk not yet added
        for (int polls = 0;;) {
            const int idx = c - lane;
            // lanes past chunk 0 read a virtual inclusive zero (chunk 0 is
            // inclusive, so the walk never needs them)
            const unsigned long long w = idx >= 0 ? load_scan_status(status + idx) : kScanInclusive;
            const uint32_t pending = __ballot_sync(0xffffffffu, (w >> 62) == 0);
            const uint32_t inclusive = __ballot_sync(0xffffffffu, (w >> 62) == 2);
            const int first_pending = pending ? __ffs(pending) - 1 : 32;
            const int first_inclusive = inclusive ? __ffs(inclusive) - 1 : 32;
            if (first_inclusive < first_pending) {
                excl += warp_sum64(lane <= first_inclusive ? static_cast<long long>(w & kScanValue) : 0);
                break;
            }
            // lanes before the first pending word are aggregates: add them and
            // continue from the pending one
            excl += warp_sum64(lane < first_pending ? static_cast<long long>(w & kScanValue) : 0);
            c -= first_pending;
            if (first_pending < 32) {
                if (++polls >= kScanPolls) {
                    if (lane == 0) atomicExch(error, 1);
                    break;
                }
                if (polls >= 32) __nanosleep(64);
            }
        }
        if (lane == 0) {
            store_scan_status(status + chunk, kScanInclusive | static_cast<unsigned long long>(excl + total));
            s_excl = excl;
        }
    }
    __syncthreads();
    const long long base = s_excl;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        tile[threadIdx.x * kScanItems + k] = static_cast<int>(base + run);
        run += v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int j = k * kScanThreads + threadIdx.x;
        const int64_t i = start + j;
        if (i < n) out[i] = tile[j];
    }
    // the chunk holding element n - 1 also writes the total
    if (threadIdx.x == 0 && start + kScanChunk >= n) out[n] = static_cast<int>(base + total);
}

// ---------------------------------------------------------------- records
// Four lanes per Gaussian walk its tile rectangle row-major; the records of one
// Gaussian are contiguous and in the same order as the reference writes them.
__global__ void __launch_bounds__(256) emit_records(const uint32_t* __restrict__ sorted_ids,
                                                    const int* __restrict__ record_start,
                                                    const int4* __restrict__ rects, int n, int tile_count_x,
                                                    uint32_t* __restrict__ tile_keys,
                                                    uint32_t* __restrict__ record_ids, int64_t capacity,
                                                    int* overflow) {
    pdl_begin();
    const int64_t gidx = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int64_t p = gidx >> 2;
    const int sub = static_cast<int>(gidx & 3);
    if (p >= n) return;
    const int begin = record_start[p];
    const int count = record_start[p + 1] - begin;
    if (count <= 0) return;
    if (begin + static_cast<int64_t>(count) > capacity) {
        if (sub == 0 && overflow) atomicExch(overflow, 1);
        if (begin >= capacity) return;
    }
    const uint32_t id = sorted_ids[p];
    const int4 r = rects[id];
    const int width = r.z - r.x;
    // past the capacity the overflow flag is set and the records that still fit
    // are written, so every slot below min(total, capacity) - all the sort and
    // the blend read - holds a record
    const int fit = static_cast<int>(min(static_cast<int64_t>(count), capacity - begin));
    for (int k = sub; k < fit; k += 4) {
        int ty = r.y + k / width;
        int tx = r.x + k % width;
        tile_keys[begin + k] = static_cast<uint32_t>(ty * tile_count_x + tx);
        record_ids[begin + k] = id;
    }
}

// Tile t's records are [offsets[t], offsets[t + 1]) of the tile-sorted keys. With
// v(-1) = -1, v(r) = the tile of record r and v(n) = tile_count, position r in
// [0, n] starts every tile in (v(r - 1), v(r)]. Each thread takes a run of
// kRangeItems consecutive positions and issues the run's loads together: two
// 16-byte loads of its eight keys plus the key before them (the previous
// thread's line), or scalar loads for the ragged tail and unaligned buffers.
constexpr int kRangeItems = 8;

// a key clamped to tile_count, so every offsets write below stays in range
__device__ __forceinline__ int range_key(uint32_t key, int tile_count) {
    return static_cast<int>(min(key, static_cast<uint32_t>(tile_count)));
}

static_assert(kRangeItems == 8, "the vector path of tile_ranges loads eight keys as two uint4");

__global__ void __launch_bounds__(256) tile_ranges(const uint32_t* __restrict__ tiles, const int* n_dev,
                                                   int max_records, int tile_count, int64_t* __restrict__ offsets) {
    pdl_begin();
    const int n = min(*n_dev, max_records);
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    const int64_t first = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (n <= 0) {
        for (int64_t i = first; i <= tile_count; i += stride) offsets[i] = 0;
        return;
    }
    const int64_t positions = static_cast<int64_t>(n) + 1;
    const bool aligned = (reinterpret_cast<uintptr_t>(tiles) & 15u) == 0;
    for (int64_t r0 = first * kRangeItems; r0 < positions; r0 += stride * kRangeItems) {
        int v[kRangeItems + 1];
        if (aligned && r0 + kRangeItems <= n) {
            // r0 is a multiple of 8, so tiles + r0 and tiles + r0 + 4 are 16-byte aligned
            const uint4 a = __ldg(reinterpret_cast<const uint4*>(tiles + r0));
            const uint4 b = __ldg(reinterpret_cast<const uint4*>(tiles + r0 + 4));
            v[0] = r0 == 0 ? -1 : range_key(__ldg(tiles + r0 - 1), tile_count);
            v[1] = range_key(a.x, tile_count);
            v[2] = range_key(a.y, tile_count);
            v[3] = range_key(a.z, tile_count);
            v[4] = range_key(a.w, tile_count);
            v[5] = range_key(b.x, tile_count);
            v[6] = range_key(b.y, tile_count);
            v[7] = range_key(b.z, tile_count);
            v[8] = range_key(b.w, tile_count);
        } else {
#pragma unroll
            for (int k = 0; k <= kRangeItems; ++k) {
                const int64_t r = r0 - 1 + k;
                v[k] = r < 0 ? -1 : r < n ? range_key(__ldg(tiles + r), tile_count) : tile_count;
            }
        }
#pragma unroll
        for (int k = 1; k <= kRangeItems; ++k) {
            const int64_t r = r0 - 1 + k;
            if (r >= positions) break;
            for (int e = v[k - 1] + 1; e <= v[k]; ++e) offsets[e] = r;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------- host side
// Words of the sort scratch for max_count pairs: four passes' digit totals
// (kTotalCopies rows of 256 each), then one 256-bin histogram per 3072-key
// block (the byte size adds 256 bytes of alignment slack).
constexpr size_t kDigitTotalWords = static_cast<size_t>(kBins) * kTotalCopies;
constexpr size_t radix_sort_scratch_words(int max_count) {
    return static_cast<size_t>(kBins) * ((static_cast<size_t>(max_count > 0 ? max_count : 1) + kSortChunk - 1) /
                                         kSortChunk) +
           kDigitTotalWords * 4;
}

size_t radix_sort_scratch_bytes(int max_count) {
    return radix_sort_scratch_words(max_count) * sizeof(uint32_t) + 256;
}

RadixSortScratch radix_sort_scratch(void* base, int max_count) {
    RadixSortScratch s;
    s.max_blocks = static_cast<size_t>(ceil_div(max_count > 0 ? max_count : 1, kSortChunk));
    s.digit_total = static_cast<uint32_t*>(base);
    s.block_hist = s.digit_total + kDigitTotalWords * 4;
    return s;
}

static int radix_sort_impl(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt,
                           bool identity_values, int max_count, const int* count_device, int begin_bit,
                           int end_bit, const RadixSortScratch& scratch, bool* result_in_alt, int* kept_device,
                           cudaStream_t stream) {
    *result_in_alt = false;
    if (max_count <= 0 || end_bit <= begin_bit) return GSN_OK;
    const int passes = (end_bit - begin_bit + 7) / 8;
    if (passes > 4 || !keys || !keys_alt || !values || !values_alt) return GSN_ERR_INVALID_ARGUMENT;
    if (cudaMemsetAsync(scratch.digit_total, 0, sizeof(uint32_t) * kDigitTotalWords * passes, stream) != cudaSuccess)
        return GSN_ERR_CUDA;
    const int blocks = ceil_div(max_count, kSortChunk);
    uint32_t *kin = keys, *vin = values, *kout = keys_alt, *vout = values_alt;
    const int* count = count_device;
    // the key bits split into passes of near-equal width (13 tile bits: 7 + 6),
    // so no pass pays for a 256-bin digit it does not need
    const int width = end_bit - begin_bit;
    int bit = begin_bit;
    for (int p = 0; p < passes; ++p) {
        const int digit_bits = width / passes + (p < width % passes ? 1 : 0);
        const uint32_t mask = (1u << digit_bits) - 1u;
        const int bins = 1 << digit_bits;
        uint32_t* dt = scratch.digit_total + kDigitTotalWords * p;
        const bool drop = kept_device && p == 0;
        if (drop)
            launch_step(radix_upsweep<true>, blocks, kSortThreads, 0, stream, kin, count, max_count, bit, mask,
                        scratch.block_hist, scratch.max_blocks, dt);
        else
            launch_step(radix_upsweep<false>, blocks, kSortThreads, 0, stream, kin, count, max_count, bit, mask,
                        scratch.block_hist, scratch.max_blocks, dt);
        launch_step(radix_scan, bins, kSortThreads, 0, stream, count, max_count, scratch.block_hist,
                    scratch.max_blocks, dt);
        const uint32_t* vsrc = identity_values && p == 0 ? nullptr : vin;
        if (identity_values && p == 0 && drop)
            launch_step(radix_downsweep<true, true>, blocks, kSortThreads, 0, stream,
                kin, vsrc, kout, vout, count, max_count, bit, mask, digit_bits, scratch.block_hist,
                scratch.max_blocks);
        else if (identity_values && p == 0)
            launch_step(radix_downsweep<true, false>, blocks, kSortThreads, 0, stream,
                kin, vsrc, kout, vout, count, max_count, bit, mask, digit_bits, scratch.block_hist,
                scratch.max_blocks);
        else if (drop)
            launch_step(radix_downsweep<false, true>, blocks, kSortThreads, 0, stream,
                kin, vsrc, kout, vout, count, max_count, bit, mask, digit_bits, scratch.block_hist,
                scratch.max_blocks);
        else
            launch_step(radix_downsweep<false, false>, blocks, kSortThreads, 0, stream,
                kin, vsrc, kout, vout, count, max_count, bit, mask, digit_bits, scratch.block_hist,
                scratch.max_blocks);
        if (drop) {
            // later passes (and the caller) see only the kept keys
            launch_step(radix_kept, 1, kBins, 0, stream, dt, kept_device);
            count = kept_device;
        }
        uint32_t* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
        bit += digit_bits;
    }
    *result_in_alt = (passes % 2) == 1;
    return launched(3 * passes + (kept_device ? 1 : 0));
}

int launch_radix_sort(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt,
                      bool identity_values, int max_count, const int* count_device, int begin_bit,
                      int end_bit, const RadixSortScratch& scratch, bool* result_in_alt,
                      cudaStream_t stream) {
    return radix_sort_impl(keys, values, keys_alt, values_alt, identity_values, max_count, count_device, begin_bit,
                           end_bit, scratch, result_in_alt, nullptr, stream);
}

int launch_radix_sort_dropping(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt,
                               bool identity_values, int max_count, const int* count_device, int begin_bit,
                               int end_bit, const RadixSortScratch& scratch, bool* result_in_alt, int* kept_device,
                               cudaStream_t stream) {
    if (!kept_device) return GSN_ERR_INVALID_ARGUMENT;
    return radix_sort_impl(keys, values, keys_alt, values_alt, identity_values, max_count, count_device, begin_bit,
                           end_bit, scratch, result_in_alt, kept_device, stream);
}

// ---------------------------------------------------------------- no-alloc sort
// Scratch of gsn_sort_pairs_noalloc: the digit totals and per-block histograms
// of the sort for up to kNoAllocMaxCount pairs, in a file-scope device array
// (5.7 MB on every GPU that loads the library, held until exit). Host code
// cannot use the array's name as a device address, so its address is looked up
// once per device with cudaGetSymbolAddress and cached; the cached address is
// that of the module loaded in the device's current context, so it does not
// survive cudaDeviceReset (the library's other entry points do not either: a
// reset frees every buffer they hold).
constexpr int kNoAllocMaxCount = 1 << 24;
constexpr size_t kNoAllocScratchWords = radix_sort_scratch_words(kNoAllocMaxCount);
static __device__ __align__(256) uint32_t g_noalloc_sort_scratch[kNoAllocScratchWords];
// the array is 256-byte aligned, so it needs the layout's words without the slack
static_assert(sizeof(g_noalloc_sort_scratch) >= radix_sort_scratch_words(kNoAllocMaxCount) * sizeof(uint32_t),
              "the no-alloc scratch array must hold the sort layout for its maximum count");

int noalloc_sort_max_count() { return kNoAllocMaxCount; }

int launch_radix_sort_noalloc(uint32_t* keys, uint32_t* values, uint32_t* keys_alt, uint32_t* values_alt, int count,
                              int begin_bit, int end_bit, bool* result_in_alt, cudaStream_t stream) {
    *result_in_alt = false;
    if (count > kNoAllocMaxCount) return GSN_ERR_CAPACITY;
    static std::mutex mutex;
    static void* scratch_address[64] = {};
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) return GSN_ERR_CUDA;
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(mutex);
        if (!scratch_address[device]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_sort_scratch) != cudaSuccess || !p) return GSN_ERR_CUDA;
            scratch_address[device] = p;
        }
        base = scratch_address[device];
    }
    // the layout for `count` pairs is a prefix of the array; the digit totals
    // are cleared by launch_radix_sort and every histogram word is written
    // before it is read, so nothing left by an earlier call is used
    RadixSortScratch scratch = radix_sort_scratch(base, count);
    return launch_radix_sort(keys, values, keys_alt, values_alt, false, count, nullptr, begin_bit, end_bit, scratch,
                             result_in_alt, stream);
}

// Scan scratch: the ticket counter and the error word (16 bytes), then one
// 64-bit look-back status word per 2048-element chunk.
size_t scan_scratch_bytes(int n) {
    return 16 + static_cast<size_t>(ceil_div(n > 0 ? n : 1, kScanChunk)) * sizeof(unsigned long long);
}

int launch_exclusive_scan(const int* in, const uint32_t* gather, int* out, int n, void* scratch,
                          cudaStream_t stream, const int* valid_device) {
    if (n < 0) return GSN_ERR_INVALID_ARGUMENT;
    if (n == 0) return cudaMemsetAsync(out, 0, sizeof(int), stream) == cudaSuccess ? GSN_OK : GSN_ERR_CUDA;
    const int blocks = ceil_div(n, kScanChunk);
    int* ticket = static_cast<int*>(scratch);
    auto* status = reinterpret_cast<unsigned long long*>(static_cast<char*>(scratch) + 16);
    if (cudaMemsetAsync(scratch, 0, scan_scratch_bytes(n), stream) != cudaSuccess) return GSN_ERR_CUDA;
    launch_step(scan_onepass, blocks, kScanThreads, 0, stream, in, gather, n, valid_device, out, status, ticket,
                ticket + 1);
    return launched(1);
}

int launch_emit_records(const uint32_t* sorted_ids, const int* record_start, const int4* rects, int n,
                        int tile_count_x, uint32_t* tile_keys, uint32_t* record_ids, int64_t capacity,
                        int* overflow, cudaStream_t stream) {
    if (n <= 0) return GSN_OK;
    launch_step(emit_records, ceil_div(4ll * n, 256), 256, 0, stream, sorted_ids, record_start, rects, n,
                tile_count_x, tile_keys, record_ids, capacity, overflow);
    return launched(1);
}

int launch_tile_ranges(const uint32_t* sorted_tiles, const int* record_count_device, int max_records,
                       int tile_count, int64_t* offsets, cudaStream_t stream) {
    const int64_t runs = ceil_div(static_cast<int64_t>(max_records) + 1, kRangeItems);
    int64_t work = runs > tile_count + 1 ? runs : tile_count + 1;
    int blocks = static_cast<int>(ceil_div(work, 256));
    if (blocks > 148 * 32) blocks = 148 * 32;
    launch_step(tile_ranges, blocks, 256, 0, stream, sorted_tiles, record_count_device, max_records, tile_count,
                offsets);
    return launched(1);
}

}  // namespace gsn
