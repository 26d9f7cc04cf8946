// Preprocess sorting: a stable LSD radix sort of (key, value) uint32 pairs
// and an exclusive scan of uint32 counts, both project-written.
//
// The binning of a trajectory needs two stable sorts by small integer keys
// (frame x tile: samples by home tile, then (tile, sample) pairs by target
// tile) and one scan (pair counts to offsets); the reference does the same
// with thrust::sort_by_key and thrust::inclusive_scan
// (cuGriddingConvolution.cu:361-422).  Stability keeps the gridding's
// per-cell summation order a function of the trajectory alone, so results
// are bit-reproducible.
//
// Radix sort: ceil(end_bit / 11) passes of equal digits of at most 11 bits
// (a 10-bit key sorts in one pass), each pass three launches over tiles of
// kSortTile elements (256 threads, 8 warps; a warp owns a contiguous run of
// kSortTile / 8 elements):
//   upsweep    per-tile digit histogram (shared-memory atomics), written
//              digit-major: hist[digit * ntiles + tile];
//   scan       exclusive scan of hist (the global position of every
//              (digit, tile) run: all tiles of digit 0 first, in tile order);
//   downsweep  per-warp digit counts, their exclusive prefix over the warps
//              of the tile, then each warp walks its run in order, 32
//              elements at a time: lanes with equal digits find each other
//              with __match_any_sync, rank by lane order, and the lowest of
//              them advances the warp's counter -- element order is kept
//              within a warp, across warps and across tiles.
// Scan: reduce each tile of kScanTile counts, scan the tile sums in one block
// (sequential over chunks), then scan each tile with its offset.
#include <algorithm>

#include "gb_internal.cuh"

namespace gb {

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *tile_scratch, cudaStream_t st);

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortPerWarp = 512;                        // 16 rounds of 32
constexpr int kSortTile = kSortWarps * kSortPerWarp;     // 4096 elements
constexpr int kMaxRadixBits = 11;

constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 16;
constexpr int kScanTile = kScanThreads * kScanPerThread;  // 4096 counts

template <int RB>
__global__ void __launch_bounds__(kSortThreads) k_radix_upsweep(const uint32_t *__restrict__ keys, int64_t n,
                                                                int shift, int64_t ntiles,
                                                                uint32_t *__restrict__ hist) {
    constexpr int R = 1 << RB;
    __shared__ uint32_t h[R];
    for (int d = threadIdx.x; d < R; d += kSortThreads) h[d] = 0u;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        const int64_t e = base + i;
        if (e < n) atomicAdd(&h[(keys[e] >> shift) & (R - 1)], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < R; d += kSortThreads) hist[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

// Shared memory: kSortWarps x 2^RB counters (dynamic, up to 64 KB).
template <int RB>
__global__ void __launch_bounds__(kSortThreads)
k_radix_downsweep(const uint32_t *__restrict__ keys_in, const uint32_t *__restrict__ vals_in,
                  uint32_t *__restrict__ keys_out, uint32_t *__restrict__ vals_out, int64_t n, int shift,
                  int64_t ntiles, const uint32_t *__restrict__ offs) {
    constexpr int R = 1 << RB;
    extern __shared__ uint32_t g_sort_cnt[];
    auto cnt = [&](int w, uint32_t d) -> uint32_t & { return g_sort_cnt[w * R + d]; };
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * R; i += kSortThreads) g_sort_cnt[i] = 0u;
    __syncthreads();
    const int64_t wbase = (int64_t)blockIdx.x * kSortTile + (int64_t)warp * kSortPerWarp;
    const uint32_t lt = (1u << lane) - 1u;
    // per-warp digit counts
    for (int r = 0; r < kSortPerWarp; r += 32) {
        const int64_t e = wbase + r + lane;
        const bool ok = e < n;
        const uint32_t d = ok ? (keys_in[e] >> shift) & (R - 1) : (uint32_t)R;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (ok && (peers & lt) == 0u) cnt(warp, d) += (uint32_t)__popc(peers);
    }
    __syncthreads();
    // global start of every (warp, digit) run of this tile
    for (int d = threadIdx.x; d < R; d += kSortThreads) {
        uint32_t run = offs[(int64_t)d * ntiles + blockIdx.x];
        for (int w = 0; w < kSortWarps; w++) {
            const uint32_t c = cnt(w, d);
            cnt(w, d) = run;
            run += c;
        }
    }
    __syncthreads();
    for (int r = 0; r < kSortPerWarp; r += 32) {
        const int64_t e = wbase + r + lane;
        const bool ok = e < n;
        uint32_t key = 0u, val = 0u;
        if (ok) {
            key = keys_in[e];
            val = vals_in[e];
        }
        const uint32_t d = ok ? (key >> shift) & (R - 1) : (uint32_t)R;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        if (ok) {
            const uint32_t pos = cnt(warp, d) + (uint32_t)__popc(peers & lt);
            keys_out[pos] = key;
            vals_out[pos] = val;
        }
        __syncwarp();
        if (ok && (peers & lt) == 0u) cnt(warp, d) += (uint32_t)__popc(peers);
        __syncwarp();
    }
}

template <int RB>
void radix_pass(const uint32_t *ki, const uint32_t *vi, uint32_t *ko, uint32_t *vo, int64_t n, int shift,
                int64_t ntiles, uint32_t *hist, uint32_t *scan_tmp, cudaStream_t st) {
    constexpr int R = 1 << RB;
    const size_t smem = (size_t)kSortWarps * R * sizeof(uint32_t);
    if (smem > 48 * 1024)   // set on every call: the attribute belongs to the current device's context
        GB_CUDA(cudaFuncSetAttribute(k_radix_downsweep<RB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    k_radix_upsweep<RB><<<(unsigned)ntiles, kSortThreads, 0, st>>>(ki, n, shift, ntiles, hist); note_launch();
    GB_CUDA(cudaGetLastError());
    exclusive_scan_u32(hist, hist, (int64_t)R * ntiles, scan_tmp, st);
    k_radix_downsweep<RB><<<(unsigned)ntiles, kSortThreads, smem, st>>>(ki, vi, ko, vo, n, shift, ntiles, hist);
    note_launch();
    GB_CUDA(cudaGetLastError());
}

// Exclusive scan of the kScanTile counts of each tile in shared memory,
// plus `offset` (tile_sums scanned) when given; tile sums out when asked.
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t s = lane < kScanThreads / 32 ? sh[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < kScanThreads / 32) sh[lane] = s;
    }
    __syncthreads();
    const uint32_t before = warp > 0 ? sh[warp - 1] : 0u;
    const uint32_t total = sh[kScanThreads / 32 - 1];
    __syncthreads();
    sh[32] = total;   // read by the caller after a barrier
    return before + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t *__restrict__ in, int64_t n,
                                                             uint32_t *__restrict__ out,
                                                             uint32_t *__restrict__ tile_sums,
                                                             const uint32_t *__restrict__ tile_offs) {
    __shared__ uint32_t sh[33];
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanPerThread;
    uint32_t v[kScanPerThread];
    uint32_t s = 0u;
#pragma unroll
    for (int i = 0; i < kScanPerThread; i++) {
        v[i] = base + i < n ? in[base + i] : 0u;
        s += v[i];
    }
    uint32_t pre = block_exclusive_scan(s, sh);
    __syncthreads();
    if (tile_sums && threadIdx.x == 0) tile_sums[blockIdx.x] = sh[32];
    if (!out) return;
    pre += tile_offs ? tile_offs[blockIdx.x] : 0u;
#pragma unroll
    for (int i = 0; i < kScanPerThread; i++) {
        if (base + i < n) out[base + i] = pre;
        pre += v[i];
    }
}

// One block: exclusive scan of a short array, tile after tile with a running
// carry (a few tiles: one launch instead of three).  In place allowed.
__global__ void __launch_bounds__(kScanThreads) k_scan_small(const uint32_t *__restrict__ in, int64_t n,
                                                             uint32_t *__restrict__ out) {
    __shared__ uint32_t sh[33];
    uint32_t carry = 0u;
    for (int64_t tb = 0; tb < n; tb += kScanTile) {
        const int64_t base = tb + (int64_t)threadIdx.x * kScanPerThread;
        uint32_t v[kScanPerThread];
        uint32_t s = 0u;
#pragma unroll
        for (int i = 0; i < kScanPerThread; i++) {
            v[i] = base + i < n ? in[base + i] : 0u;
            s += v[i];
        }
        uint32_t pre = block_exclusive_scan(s, sh);
        __syncthreads();
        const uint32_t total = sh[32];
        pre += carry;
#pragma unroll
        for (int i = 0; i < kScanPerThread; i++) {
            if (base + i < n) out[base + i] = pre;
            pre += v[i];
        }
        carry += total;
        __syncthreads();
    }
}

// One block: exclusive scan of the tile sums, chunk by chunk.
__global__ void __launch_bounds__(kScanThreads) k_scan_sums(uint32_t *__restrict__ sums, int64_t n) {
    __shared__ uint32_t sh[33];
    uint32_t carry = 0u;
    for (int64_t c = 0; c < n; c += kScanThreads) {
        const int64_t i = c + threadIdx.x;
        const uint32_t v = i < n ? sums[i] : 0u;
        const uint32_t pre = block_exclusive_scan(v, sh);
        __syncthreads();
        const uint32_t total = sh[32];
        if (i < n) sums[i] = carry + pre;
        carry += total;
        __syncthreads();
    }
}

}  // namespace

void scan_scratch_need(int64_t n, size_t *bytes) {
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    *bytes = (size_t)std::max<int64_t>(tiles, 1) * sizeof(uint32_t);
}

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *tile_scratch, cudaStream_t st) {
    if (n <= 0) return;
    const int64_t tiles = (n + kScanTile - 1) / kScanTile;
    if (tiles <= 4) {   // short: one block, one launch
        k_scan_small<<<1, kScanThreads, 0, st>>>(in, n, out); note_launch();
        GB_CUDA(cudaGetLastError());
        return;
    }
    k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, nullptr, tile_scratch, nullptr); note_launch();
    GB_CUDA(cudaGetLastError());
    k_scan_sums<<<1, kScanThreads, 0, st>>>(tile_scratch, tiles); note_launch();
    GB_CUDA(cudaGetLastError());
    k_scan_tiles<<<(unsigned)tiles, kScanThreads, 0, st>>>(in, n, out, nullptr, tile_scratch); note_launch();
    GB_CUDA(cudaGetLastError());
}

void exclusive_scan(const uint32_t *in, uint32_t *out, int64_t n, DevBuf<unsigned char> &tmp, cudaStream_t st) {
    size_t bytes = 0;
    scan_scratch_need(n, &bytes);
    tmp.ensure(bytes);
    exclusive_scan_u32(in, out, n, reinterpret_cast<uint32_t *>(tmp.get()), st);
}

void sort_pairs(const uint32_t *keys_in, uint32_t *keys_out, const uint32_t *vals_in, uint32_t *vals_out, int64_t n,
                int end_bit, DevBuf<unsigned char> &tmp, cudaStream_t st) {
    if (n <= 0) return;
    if (n >= (1ll << 31)) fail(GB_ERR_INVALID_ARGUMENT, "sort of 2^31 or more elements");
    end_bit = std::max(1, std::min(end_bit, 32));
    const int passes = (end_bit + kMaxRadixBits - 1) / kMaxRadixBits;
    const int rb = std::max(4, (end_bit + passes - 1) / passes);   // digit bits, 4..11
    const int64_t ntiles = (n + kSortTile - 1) / kSortTile;
    const int64_t nhist = ntiles << rb;
    size_t scan_bytes = 0;
    scan_scratch_need(nhist, &scan_bytes);
    // layout: hist [nhist] | scan scratch | two ping-pong (key, value) arrays
    const size_t hist_bytes = ((size_t)nhist * sizeof(uint32_t) + 255) & ~(size_t)255;
    scan_bytes = (scan_bytes + 255) & ~(size_t)255;
    const size_t arr_bytes = (((size_t)n * sizeof(uint32_t)) + 255) & ~(size_t)255;
    const int nbuf = passes > 2 ? 2 : (passes == 2 ? 1 : 0);
    tmp.ensure(hist_bytes + scan_bytes + (size_t)nbuf * 2 * arr_bytes);
    unsigned char *b = tmp.get();
    uint32_t *hist = reinterpret_cast<uint32_t *>(b);
    uint32_t *scan_tmp = reinterpret_cast<uint32_t *>(b + hist_bytes);
    uint32_t *pk[2], *pv[2];
    for (int i = 0; i < 2; i++) {
        pk[i] = reinterpret_cast<uint32_t *>(b + hist_bytes + scan_bytes + (size_t)(2 * i) * arr_bytes);
        pv[i] = reinterpret_cast<uint32_t *>(b + hist_bytes + scan_bytes + (size_t)(2 * i + 1) * arr_bytes);
    }
    const uint32_t *ki = keys_in, *vi = vals_in;
    for (int p = 0; p < passes; p++) {
        const int shift = rb * p;
        uint32_t *ko, *vo;
        if (p == passes - 1) {
            ko = keys_out;
            vo = vals_out;
        } else {
            ko = pk[p & 1];
            vo = pv[p & 1];
        }
        switch (rb) {
        case 4: radix_pass<4>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        case 5: radix_pass<5>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        case 6: radix_pass<6>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        case 7: radix_pass<7>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        case 8: radix_pass<8>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        case 9: radix_pass<9>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        case 10: radix_pass<10>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        default: radix_pass<11>(ki, vi, ko, vo, n, shift, ntiles, hist, scan_tmp, st); break;
        }
        ki = ko;
        vi = vo;
    }
}

}  // namespace gb
