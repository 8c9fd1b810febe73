// sort.cu -- stable LSD radix sort of particle keys and device-wide scans.
//
// Replaces the reference's unordered global atomics (src/mpm_solver3d.cu:
// 277-286): particles are ordered by (block, cell) key every step so that the
// P2G scatter can be done per block in a fixed order.  The sort is stable
// (ties keep their previous order), hence bit-exact and deterministic.
//
// Per 8-bit digit: upsweep (per-tile digit histogram), exclusive scan of the
// digit-major histogram, downsweep (warp match_any ranking, stable scatter).
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine_host.hpp"

namespace mpm {

namespace {

constexpr int kScanItems = 16;                      // per thread
constexpr int kScanChunk = kThreads * kScanItems;   // 4096 per CTA
constexpr int kSortItems = kSortTileKeys / kThreads;
constexpr int kSortTile = kSortTileKeys;

template <class T>
__device__ __forceinline__ T warpInclusiveScan(T x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Exclusive scan across the 256 threads of a CTA; returns the CTA total in *total.
template <class T>
__device__ __forceinline__ T blockExclusiveScan(T x, T* total) {
    __shared__ T warp_tot[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warpInclusiveScan(x);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T t = lane < kWarps ? warp_tot[lane] : T(0);
        T ti = warpInclusiveScan(t);
        if (lane < kWarps) warp_tot[lane] = ti - t;
        // CTA total: inclusive value at the last warp
        T tl = __shfl_sync(0xffffffffu, ti, kWarps - 1);
        if (lane == 0) *total = tl;
    }
    __syncthreads();
    T r = inc - x + warp_tot[warp];
    __syncthreads();
    return r;
}

template <class T>
__global__ void __launch_bounds__(kThreads) scanReduceKernel(const T* in, size_t n, T* partials) {
    size_t base = (size_t)blockIdx.x * kScanChunk;
    T s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        size_t i = base + (size_t)j * kThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    __shared__ T tot;
    (void)blockExclusiveScan(s, &tot);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

// Single CTA exclusive scan of up to kScanChunk partials; writes the grand
// total to *total (if non-null).
template <class T>
__global__ void __launch_bounds__(kThreads) scanPartialsKernel(T* partials, int m, T* total) {
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        int i = threadIdx.x * kScanItems + j;
        v[j] = i < m ? partials[i] : T(0);
        s += v[j];
    }
    __shared__ T tot;
    T run = blockExclusiveScan(s, &tot);
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        int i = threadIdx.x * kScanItems + j;
        if (i < m) partials[i] = run;
        run += v[j];
    }
    if (threadIdx.x == 0 && total) *total = tot;
}

template <class T>
__global__ void __launch_bounds__(kThreads) scanDownsweepKernel(const T* in, T* out, size_t n, const T* partials) {
    size_t base = (size_t)blockIdx.x * kScanChunk + (size_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T s = 0;
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        size_t i = base + j;
        v[j] = i < n ? in[i] : T(0);
        s += v[j];
    }
    __shared__ T tot;
    T run = blockExclusiveScan(s, &tot) + partials[blockIdx.x];
#pragma unroll
    for (int j = 0; j < kScanItems; ++j) {
        size_t i = base + j;
        if (i < n) out[i] = run;
        run += v[j];
    }
}

// --- radix sort -------------------------------------------------------------

__global__ void __launch_bounds__(kThreads) radixUpsweepKernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                int shift, uint32_t mask, uint32_t* __restrict__ hist,
                                                                int ntiles) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    size_t base = (size_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int j = 0; j < kSortItems; ++j) {
        size_t i = base + (size_t)j * kThreads + threadIdx.x;
        bool valid = i < n;
        uint32_t d = valid ? (keys[i] >> shift) & mask : 0xffffffffu;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        int leader = __ffs(peers) - 1;
        if (valid && lane == leader) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

template <bool kIdentVals>
__global__ void __launch_bounds__(kThreads) radixDownsweepKernel(const uint32_t* __restrict__ keys_in,
                                                                  const uint32_t* __restrict__ vals_in,
                                                                  uint32_t* __restrict__ keys_out,
                                                                  uint32_t* __restrict__ vals_out,
                                                                  const uint32_t* __restrict__ offsets, uint32_t n,
                                                                  int shift, uint32_t mask, int ntiles) {
    __shared__ uint32_t cnt[kWarps][256];
    for (int i = threadIdx.x; i < kWarps * 256; i += kThreads) (&cnt[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const size_t base = (size_t)blockIdx.x * kSortTile + (size_t)warp * 32 * kSortItems;
    uint32_t k[kSortItems], v[kSortItems], r[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        size_t i = base + (size_t)j * 32 + lane;
        bool valid = i < n;
        k[j] = valid ? keys_in[i] : 0u;
        v[j] = valid ? (kIdentVals ? (uint32_t)i : vals_in[i]) : 0u;
        uint32_t d = valid ? (k[j] >> shift) & mask : 256u;
        uint32_t peers = __match_any_sync(0xffffffffu, d);
        int leader = __ffs(peers) - 1;
        uint32_t before = valid ? cnt[warp][d] : 0u;
        r[j] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == leader) cnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            uint32_t c = cnt[w][threadIdx.x];
            cnt[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        size_t i = base + (size_t)j * 32 + lane;
        if (i < n) {
            uint32_t d = (k[j] >> shift) & mask;
            uint32_t pos = offsets[(size_t)d * ntiles + blockIdx.x] + cnt[warp][d] + r[j];
            keys_out[pos] = k[j];
            vals_out[pos] = v[j];
        }
    }
}

// --- single-pass ("onesweep") radix passes -----------------------------------
//
// One kernel counts the digits of every pass over all keys; then each pass is
// one kernel: a CTA takes the next tile (dynamic tile ids, so tile t only
// ever waits on tiles that started earlier), ranks its keys stably, publishes
// its per-digit count, and finds the count of every earlier tile with the
// same digit by looking back over their published words.  A word holds a
// 2-bit flag (aggregate / inclusive prefix) and a 30-bit count.  Every wait
// is bounded: after kLookbackLimit polls the kernel raises an error flag and
// goes on instead of spinning forever.

constexpr uint32_t kFlagAgg = 1u << 30, kFlagPrefix = 2u << 30, kCountMask = (1u << 30) - 1u;
constexpr int kLookbackLimit = 1 << 22;
constexpr int kLookWidth = 8;  // predecessor words read per look-back round trip

__global__ void __launch_bounds__(kThreads) onesweepHistKernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                const uint32_t* __restrict__ n_dev, int passes,
                                                                int bits, uint32_t* __restrict__ ghist) {
    if (n_dev) n = *n_dev;  // the key count is only known on the device
    __shared__ uint32_t h[4][256];
    for (int i = threadIdx.x; i < 4 * 256; i += kThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const size_t stride = (size_t)gridDim.x * kThreads;
    const size_t n_round = ((size_t)n + 31) / 32 * 32;  // whole warps iterate together
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < n_round; i += stride) {
        const bool valid = i < n;
        const uint32_t key = valid ? keys[i] : 0u;
        for (int p = 0; p < passes; ++p) {
            const int shift = 8 * p;
            const int pb = bits - shift < 8 ? bits - shift : 8;
            const uint32_t mask = (1u << (pb > 0 ? pb : 1)) - 1u;
            const uint32_t d = valid ? (key >> shift) & mask : 0xffffffffu;
            const uint32_t peers = __match_any_sync(0xffffffffu, d);
            if (valid && lane == __ffs(peers) - 1) atomicAdd(&h[p][d], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kThreads)
        if ((&h[0][0])[i]) atomicAdd(&ghist[i], (&h[0][0])[i]);
}

template <bool kIdentVals>
__global__ void __launch_bounds__(kThreads, 4) onesweepPassKernel(const uint32_t* __restrict__ keys_in,
                                                                const uint32_t* __restrict__ vals_in,
                                                                uint32_t* __restrict__ keys_out,
                                                                uint32_t* __restrict__ vals_out, uint32_t n,
                                                                const uint32_t* __restrict__ n_dev,
                                                                int shift, uint32_t mask,
                                                                const uint32_t* __restrict__ ghist,
                                                                uint32_t* __restrict__ tile_counter,
                                                                uint32_t* __restrict__ status,
                                                                uint32_t* __restrict__ err) {
    __shared__ uint32_t cnt[kWarps][256];
    __shared__ uint32_t base[256];
    __shared__ uint32_t tile_s;
    __shared__ uint32_t tot;
    for (int i = threadIdx.x; i < kWarps * 256; i += kThreads) (&cnt[0][0])[i] = 0;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
    {   // global start of every digit: exclusive scan of this pass's digit counts
        const uint32_t g = ghist[threadIdx.x];
        base[threadIdx.x] = blockExclusiveScan(g, &tot);
    }
    __syncthreads();
    const uint32_t tile = tile_s;
    // With a device-side count the grid covers the largest possible count;
    // tiles past the actual keys leave at once (later tiles never wait on them).
    if (n_dev) n = *n_dev;
    if ((size_t)tile * kSortTile >= n) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    const size_t tbase = (size_t)tile * kSortTile + (size_t)warp * 32 * kSortItems;
    uint32_t k[kSortItems], v[kSortItems], r[kSortItems];
    // all loads first, so that they are in flight together (the ranking
    // below synchronises the warp after every item)
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const size_t i = tbase + (size_t)j * 32 + lane;
        const bool valid = i < n;
        k[j] = valid ? keys_in[i] : 0u;
        v[j] = valid ? (kIdentVals ? (uint32_t)i : vals_in[i]) : 0u;
    }
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const size_t i = tbase + (size_t)j * 32 + lane;
        const bool valid = i < n;
        const uint32_t d = valid ? (k[j] >> shift) & mask : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const int leader = __ffs(peers) - 1;
        const uint32_t before = valid ? cnt[warp][d] : 0u;
        r[j] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == leader) cnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    {
        const int d = threadIdx.x;
        uint32_t run = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            const uint32_t c = cnt[w][d];
            cnt[w][d] = run;
            run += c;
        }
        uint32_t* mine = status + (size_t)tile * 256 + d;
        uint32_t excl = 0;
        if (tile == 0) {
            atomicExch(mine, kFlagPrefix | run);
        } else {
            atomicExch(mine, kFlagAgg | run);
            // Walk back over the earlier tiles' words, kLookWidth per round
            // trip (independent loads), until an inclusive prefix is found.
            int t = (int)tile - 1;
            int polls = 0;
            bool done = false;
            while (!done && t >= 0) {
                uint32_t w[kLookWidth];
#pragma unroll
                for (int q = 0; q < kLookWidth; ++q)
                    w[q] = (t - q >= 0) ? *(volatile const uint32_t*)(status + (size_t)(t - q) * 256 + d) : kFlagPrefix;
                bool waiting = false;
#pragma unroll
                for (int q = 0; q < kLookWidth; ++q) {
                    if (done || waiting) continue;
                    const uint32_t f = w[q] & ~kCountMask;
                    if (f == 0) {  // not published yet: poll again from this tile
                        waiting = true;
                        continue;
                    }
                    excl += w[q] & kCountMask;
                    --t;
                    if (f == kFlagPrefix) done = true;
                }
                if (waiting) {
                    if (++polls > kLookbackLimit) {  // never expected: give up instead of hanging
                        atomicOr(err, 8u);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            atomicExch(mine, kFlagPrefix | (excl + run));
        }
        base[d] += excl;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; ++j) {
        const size_t i = tbase + (size_t)j * 32 + lane;
        if (i < n) {
            const uint32_t d = (k[j] >> shift) & mask;
            const uint32_t pos = base[d] + cnt[warp][d] + r[j];
            keys_out[pos] = k[j];
            vals_out[pos] = v[j];
        }
    }
}

__global__ void __launch_bounds__(kThreads) clearRangesKernel(ClearRanges r) {
    const size_t stride = (size_t)gridDim.x * kThreads;
    const size_t t = (size_t)blockIdx.x * kThreads + threadIdx.x;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        for (size_t i = t; i < r.n[k]; i += stride) r.p[k][i] = 0u;
}

}  // namespace

// A grid-stride clear: four CTAs of 256 threads per SM of a B200 cover the
// largest range (a few MB) in one or two passes.
constexpr size_t kClearMaxBlocks = 148 * 4;

void launchClear(const ClearRanges& r, cudaStream_t st) {
    size_t most = 0;
    for (int k = 0; k < 4; ++k) most = std::max(most, r.p[k] ? r.n[k] : 0);
    if (most == 0) return;
    ClearRanges q = r;
    for (int k = 0; k < 4; ++k)
        if (!q.p[k]) q.n[k] = 0;
    noteLaunches(1);
    const unsigned blocks = (unsigned)std::min<size_t>((most + kThreads - 1) / kThreads, kClearMaxBlocks);
    clearRangesKernel<<<blocks, kThreads, 0, st>>>(q);
}

// ---------------------------------------------------------------------------
// Host wrappers.
// ---------------------------------------------------------------------------
size_t onesweepScratchWords(size_t n, int bits) {
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    return (size_t)passes * 256 + 32 + (size_t)passes * radixTiles(n) * 256;
}

// Stable sort of (keys_a, identity values) by the low `bits` bits, one kernel
// per 8-bit pass.  `scratch` holds onesweepScratchWords(n, bits) words and is
// cleared here.  `err` receives bit 8 if a look-back wait gave up.  With
// `n_dev` the sort covers the first *n_dev keys (known on the device only, at
// most n) and sorts (keys_a, vals_a) pairs instead of identity values.
cudaError_t radixSortOnesweep(uint32_t* keys_a, uint32_t* vals_a, uint32_t* keys_b, uint32_t* vals_b, size_t n,
                              int bits, uint32_t* scratch, uint32_t* err, bool* result_in_b, cudaStream_t st,
                              const uint32_t* n_dev) {
    *result_in_b = false;
    if (n == 0) return cudaSuccess;
    if (n > kCountMask) return cudaErrorInvalidValue;
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    const int ntiles = (int)radixTiles(n);
    uint32_t* ghist = scratch;
    uint32_t* counters = scratch + (size_t)passes * 256;
    uint32_t* status = counters + 32;
    {
        ClearRanges cr;
        cr.p[0] = scratch;
        cr.n[0] = onesweepScratchWords(n, bits);
        launchClear(cr, st);
    }
    // ~4 keys per thread: the histogram is bound by each thread's serial
    // chain of match/atomic rounds, not by the per-block flush (1M keys:
    // 16 keys per thread 0.072 ms for the whole sort, 4 keys 0.065 ms)
    const int hblocks = (int)std::min<size_t>((n + kThreads * 4 - 1) / (kThreads * 4), 148 * 8);
    noteLaunches(1 + passes);
    onesweepHistKernel<<<hblocks, kThreads, 0, st>>>(keys_a, (uint32_t)n, n_dev, passes, bits, ghist);
    uint32_t *kin = keys_a, *vin = vals_a, *kout = keys_b, *vout = vals_b;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        int pass_bits = bits - shift < 8 ? bits - shift : 8;
        if (pass_bits <= 0) pass_bits = 1;
        const uint32_t mask = (1u << pass_bits) - 1u;
        uint32_t* stat = status + (size_t)p * ntiles * 256;
        if (p == 0 && !n_dev)
            onesweepPassKernel<true><<<ntiles, kThreads, 0, st>>>(kin, vin, kout, vout, (uint32_t)n, n_dev, shift,
                                                                  mask, ghist + 256 * p, counters + p, stat, err);
        else
            onesweepPassKernel<false><<<ntiles, kThreads, 0, st>>>(kin, vin, kout, vout, (uint32_t)n, n_dev, shift,
                                                                   mask, ghist + 256 * p, counters + p, stat, err);
        std::swap(kin, kout);
        std::swap(vin, vout);
        *result_in_b = !*result_in_b;
    }
    return cudaGetLastError();
}

size_t scanScratchElems(size_t n) { return (n + kScanChunk - 1) / kScanChunk; }

template <class T>
cudaError_t exclusiveScan(const T* in, T* out, size_t n, T* partials, T* total, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    size_t chunks = (n + kScanChunk - 1) / kScanChunk;
    if (chunks > (size_t)kScanChunk) return cudaErrorInvalidValue;
    noteLaunches(3);
    scanReduceKernel<T><<<(unsigned)chunks, kThreads, 0, st>>>(in, n, partials);
    scanPartialsKernel<T><<<1, kThreads, 0, st>>>(partials, (int)chunks, total);
    scanDownsweepKernel<T><<<(unsigned)chunks, kThreads, 0, st>>>(in, out, n, partials);
    return cudaGetLastError();
}

template cudaError_t exclusiveScan<uint32_t>(const uint32_t*, uint32_t*, size_t, uint32_t*, uint32_t*, cudaStream_t);
template cudaError_t exclusiveScan<unsigned long long>(const unsigned long long*, unsigned long long*, size_t,
                                                        unsigned long long*, unsigned long long*, cudaStream_t);

size_t radixTiles(size_t n) { return (n + kSortTile - 1) / kSortTile; }

// Same sort with every buffer supplied by the caller: `in_keys` is only read,
// the result always lands in (out_keys, out_vals), and (tmp_keys, tmp_vals)
// is the other ping-pong pair.  The pass count decides which pair the first
// pass writes so that the last pass writes the output pair.
cudaError_t radixSortPairsInto(const uint32_t* in_keys, uint32_t* out_keys, uint32_t* out_vals, uint32_t* tmp_keys,
                               uint32_t* tmp_vals, size_t n, int bits, uint32_t* hist, uint32_t* scan_partials,
                               cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    const int ntiles = (int)radixTiles(n);
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    uint32_t* dk[2] = {out_keys, tmp_keys};
    uint32_t* dv[2] = {out_vals, tmp_vals};
    int dst = (passes % 2 == 1) ? 0 : 1;
    const uint32_t* kin = in_keys;
    const uint32_t* vin = nullptr;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        int pass_bits = bits - shift < 8 ? bits - shift : 8;
        if (pass_bits <= 0) pass_bits = 1;
        const uint32_t mask = (1u << pass_bits) - 1u;
        noteLaunches(2);
        radixUpsweepKernel<<<ntiles, kThreads, 0, st>>>(kin, (uint32_t)n, shift, mask, hist, ntiles);
        cudaError_t e = exclusiveScan<uint32_t>(hist, hist, (size_t)256 * ntiles, scan_partials, nullptr, st);
        if (e != cudaSuccess) return e;
        if (p == 0)
            radixDownsweepKernel<true><<<ntiles, kThreads, 0, st>>>(kin, nullptr, dk[dst], dv[dst], hist, (uint32_t)n,
                                                                    shift, mask, ntiles);
        else
            radixDownsweepKernel<false><<<ntiles, kThreads, 0, st>>>(kin, vin, dk[dst], dv[dst], hist, (uint32_t)n,
                                                                     shift, mask, ntiles);
        kin = dk[dst];
        vin = dv[dst];
        dst ^= 1;
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Incremental sort.  Between two steps most particles keep their cell key.
// The live particle order is the previous step's sorted order, so the keys
// that did not change ("stayers") already appear in ascending order; only the
// particles whose key changed ("movers") need sorting.  Steps:
//   1. partition (one pass, look-back over tiles): stayers (key, index) and
//      movers (key, index), both in live order;
//   2. radix-sort the movers by key (stable: ties stay in index order);
//   3. merge the two sequences by (key, index).
// Every sequence is ordered by (key, live index), so the result is exactly
// the stable sort of all keys: the same keys and permutation as
// radixSortOnesweep.
// ---------------------------------------------------------------------------
namespace {

constexpr int kPartItems = 8;                        // consecutive keys per thread
constexpr int kPartTile = kThreads * kPartItems;     // 2048
constexpr int kMergeItems = 8;
constexpr int kMergeTile = kThreads * kMergeItems;   // outputs per CTA

// One tile of kPartTile keys: item j * kThreads + threadIdx.x of the tile is
// this thread's j-th (coalesced loads and stores).  A key is a mover if it
// differs from the previous step's key at the same position.  Movers keep
// their order in b, stayers in a: the rank of an item among the movers of
// its tile comes from per-warp ballots and one scan over (round, warp) in
// item order, the tile's offset from the decoupled look-back.
__global__ void __launch_bounds__(kThreads) moverPartitionKernel(
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ prev, uint32_t n, uint32_t* __restrict__ a_keys,
    uint32_t* __restrict__ a_idx, uint32_t* __restrict__ b_keys, uint32_t* __restrict__ b_idx,
    uint32_t* __restrict__ m_out, uint32_t* __restrict__ tile_counter, uint32_t* __restrict__ status, uint32_t ntiles,
    uint32_t* __restrict__ err) {
    constexpr int kW = kThreads / 32;
    __shared__ uint32_t tile_s, excl_s;
    __shared__ uint32_t wcnt[kPartItems * kW];  // movers per (round, warp), then their exclusive scan
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = tile_s;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t t0 = (size_t)tile * kPartTile;
    uint32_t k[kPartItems], ball[kPartItems];
#pragma unroll
    for (int j = 0; j < kPartItems; ++j) {
        const size_t i = t0 + (size_t)j * kThreads + threadIdx.x;
        const bool valid = i < n;
        k[j] = valid ? keys[i] : 0u;
        const uint32_t pk = valid ? prev[i] : 0u;
        ball[j] = __ballot_sync(0xffffffffu, valid && k[j] != pk);
        if (lane == 0) wcnt[j * kW + warp] = (uint32_t)__popc(ball[j]);
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the kPartItems * kW counts, in item order
        static_assert(kPartItems * kW == 64, "two counts per lane");
        const uint32_t c0 = wcnt[2 * lane], c1 = wcnt[2 * lane + 1];
        uint32_t x = c0 + c1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, x, 31);
        wcnt[2 * lane] = x - c0 - c1;
        wcnt[2 * lane + 1] = x - c1;
        if (lane == 0) {
            uint32_t excl = 0;
            if (tile == 0) {
                atomicExch(&status[0], kFlagPrefix | tot);
            } else {
                atomicExch(&status[tile], kFlagAgg | tot);
                // kLookWidth predecessor words per round trip, as in the radix passes
                int t = (int)tile - 1;
                int polls = 0;
                bool done = false;
                while (!done && t >= 0) {
                    uint32_t w[kLookWidth];
#pragma unroll
                    for (int q = 0; q < kLookWidth; ++q)
                        w[q] = (t - q >= 0) ? *(volatile const uint32_t*)(status + (t - q)) : kFlagPrefix;
                    bool waiting = false;
#pragma unroll
                    for (int q = 0; q < kLookWidth; ++q) {
                        if (done || waiting) continue;
                        const uint32_t f = w[q] & ~kCountMask;
                        if (f == 0) {  // not published yet: poll again from this tile
                            waiting = true;
                            continue;
                        }
                        excl += w[q] & kCountMask;
                        --t;
                        if (f == kFlagPrefix) done = true;
                    }
                    if (waiting) {
                        if (++polls > kLookbackLimit) {  // never expected: give up instead of hanging
                            atomicOr(err, 8u);
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                atomicExch(&status[tile], kFlagPrefix | (excl + tot));
            }
            excl_s = excl;
            if (tile == ntiles - 1) *m_out = excl + tot;
        }
    }
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kPartItems; ++j) {
        const size_t i = t0 + (size_t)j * kThreads + threadIdx.x;
        if (i >= n) break;
        const uint32_t mb = excl_s + wcnt[j * kW + warp] + (uint32_t)__popc(ball[j] & lt);  // movers before it
        if (ball[j] >> lane & 1u) {
            b_keys[mb] = k[j];
            b_idx[mb] = (uint32_t)i;
        } else {
            const uint32_t pa = (uint32_t)i - mb;  // stayers before it
            a_keys[pa] = k[j];
            a_idx[pa] = (uint32_t)i;
        }
    }
}

__device__ __forceinline__ unsigned long long composite(uint32_t key, uint32_t idx) {
    return ((unsigned long long)key << 32) | idx;
}

// Number of stayers among the first d outputs of the merge (merge path).
__device__ __forceinline__ uint32_t mergePath(const uint32_t* a_keys, const uint32_t* a_idx, uint32_t na,
                                              const uint32_t* b_keys, const uint32_t* b_idx, uint32_t nb, uint32_t d) {
    uint32_t lo = d > nb ? d - nb : 0u, hi = d < na ? d : na;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t bj = d - 1 - mid;
        if (composite(a_keys[mid], a_idx[mid]) < composite(b_keys[bj], b_idx[bj])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Split points of the merge: split[c] = stayers among the first c * kMergeTile outputs.
__global__ void __launch_bounds__(kThreads) mergeSplitKernel(const uint32_t* __restrict__ a_keys,
                                                              const uint32_t* __restrict__ a_idx,
                                                              const uint32_t* __restrict__ b_keys,
                                                              const uint32_t* __restrict__ b_idx, uint32_t n,
                                                              const uint32_t* __restrict__ m_dev,
                                                              uint32_t* __restrict__ split, uint32_t nsplit) {
    const uint32_t c = blockIdx.x * kThreads + threadIdx.x;
    if (c >= nsplit) return;
    const uint32_t m = *m_dev, na = n - m;
    const uint32_t d = (uint32_t)min((size_t)c * kMergeTile, (size_t)n);
    split[c] = mergePath(a_keys, a_idx, na, b_keys, b_idx, m, d);
}

// One CTA merges kMergeTile outputs: its stayer and mover ranges are staged in
// shared memory, each thread finds its own split there and merges 8 outputs
// into a shared output tile, which the CTA then stores with unit stride.
__global__ void __launch_bounds__(kThreads) mergeKernel(const uint32_t* __restrict__ a_keys,
                                                         const uint32_t* __restrict__ a_idx,
                                                         const uint32_t* __restrict__ b_keys,
                                                         const uint32_t* __restrict__ b_idx, uint32_t n,
                                                         const uint32_t* __restrict__ m_dev,
                                                         const uint32_t* __restrict__ split,
                                                         uint32_t* __restrict__ out_keys,
                                                         uint32_t* __restrict__ out_perm) {
    __shared__ unsigned long long sa[kMergeTile], sb[kMergeTile];
    __shared__ uint32_t ok[kMergeTile], op[kMergeTile];
    const uint32_t d0 = blockIdx.x * kMergeTile;
    if (d0 >= n) return;
    const uint32_t d1 = min(n, d0 + (uint32_t)kMergeTile);
    const uint32_t a0 = split[blockIdx.x], a1 = split[blockIdx.x + 1];
    const uint32_t b0 = d0 - a0, b1 = d1 - a1;
    const uint32_t la = a1 - a0, lb = b1 - b0;  // la + lb = d1 - d0 <= kMergeTile
    for (uint32_t i = threadIdx.x; i < la; i += kThreads) sa[i] = composite(a_keys[a0 + i], a_idx[a0 + i]);
    for (uint32_t i = threadIdx.x; i < lb; i += kThreads) sb[i] = composite(b_keys[b0 + i], b_idx[b0 + i]);
    __syncthreads();
    const uint32_t dl = threadIdx.x * kMergeItems;
    if (dl < la + lb) {
        uint32_t lo = dl > lb ? dl - lb : 0u, hi = dl < la ? dl : la;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (sa[mid] < sb[dl - 1 - mid]) lo = mid + 1;
            else hi = mid;
        }
        uint32_t ia = lo, ib = dl - lo;
        const uint32_t dend = min(dl + (uint32_t)kMergeItems, la + lb);
        for (uint32_t dd = dl; dd < dend; ++dd) {
            const bool takeA = ib >= lb || (ia < la && sa[ia] < sb[ib]);
            const unsigned long long v = takeA ? sa[ia++] : sb[ib++];
            ok[dd] = (uint32_t)(v >> 32);
            op[dd] = (uint32_t)v;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < la + lb; i += kThreads) {
        out_keys[d0 + i] = ok[i];
        out_perm[d0 + i] = op[i];
    }
    (void)m_dev;
}

}  // namespace

// Scratch layout (u32 words): a_keys, a_idx, b_keys, b_idx, b_keys2, b_idx2
// (n each), mover count, partition tile counter and status words, merge
// split points, then the movers' radix-sort scratch.
static size_t partitionTiles(size_t n) { return (n + kPartTile - 1) / kPartTile; }
static size_t mergeSplits(size_t n) { return (n + kMergeTile - 1) / kMergeTile + 1; }

size_t incrementalSortScratchWords(size_t n, int bits) {
    return 6 * n + 2 + partitionTiles(n) + mergeSplits(n) + onesweepScratchWords(n, bits) + 64;
}

cudaError_t incrementalSort(const uint32_t* keys, const uint32_t* prev, size_t n, int bits, uint32_t* out_keys,
                            uint32_t* out_perm, uint32_t* scratch, uint32_t* err, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    if (n > kCountMask) return cudaErrorInvalidValue;
    uint32_t* a_keys = scratch;
    uint32_t* a_idx = a_keys + n;
    uint32_t* b_keys = a_idx + n;
    uint32_t* b_idx = b_keys + n;
    uint32_t* b_keys2 = b_idx + n;
    uint32_t* b_idx2 = b_keys2 + n;
    uint32_t* m_dev = b_idx2 + n;
    uint32_t* tile_counter = m_dev + 1;
    uint32_t* status = tile_counter + 1;
    const size_t ptiles = partitionTiles(n);
    uint32_t* split = status + ptiles;
    const size_t nsplit = mergeSplits(n);
    uint32_t* sort_scratch = split + nsplit;
    {
        ClearRanges cr;
        cr.p[0] = m_dev;
        cr.n[0] = 2 + ptiles;
        launchClear(cr, st);
    }
    cudaError_t e = cudaSuccess;
    noteLaunches(3);
    moverPartitionKernel<<<(unsigned)ptiles, kThreads, 0, st>>>(keys, prev, (uint32_t)n, a_keys, a_idx, b_keys, b_idx,
                                                                m_dev, tile_counter, status, (uint32_t)ptiles, err);
    bool inB = false;
    e = radixSortOnesweep(b_keys, b_idx, b_keys2, b_idx2, n, bits, sort_scratch, err, &inB, st, m_dev);
    if (e != cudaSuccess) return e;
    const uint32_t* mk = inB ? b_keys2 : b_keys;
    const uint32_t* mi = inB ? b_idx2 : b_idx;
    mergeSplitKernel<<<(unsigned)((nsplit + kThreads - 1) / kThreads), kThreads, 0, st>>>(
        a_keys, a_idx, mk, mi, (uint32_t)n, m_dev, split, (uint32_t)nsplit);
    mergeKernel<<<(unsigned)(nsplit - 1), kThreads, 0, st>>>(a_keys, a_idx, mk, mi, (uint32_t)n, m_dev, split, out_keys,
                                                             out_perm);
    return cudaGetLastError();
}

}  // namespace mpm
