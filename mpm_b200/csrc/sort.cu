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
                                                                int passes, int bits, uint32_t* __restrict__ ghist) {
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
__global__ void __launch_bounds__(kThreads) onesweepPassKernel(const uint32_t* __restrict__ keys_in,
                                                                const uint32_t* __restrict__ vals_in,
                                                                uint32_t* __restrict__ keys_out,
                                                                uint32_t* __restrict__ vals_out, uint32_t n,
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

}  // namespace

// ---------------------------------------------------------------------------
// Host wrappers.
// ---------------------------------------------------------------------------
size_t onesweepScratchWords(size_t n, int bits) {
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    return (size_t)passes * 256 + 32 + (size_t)passes * radixTiles(n) * 256;
}

// Stable sort of (keys_a, identity values) by the low `bits` bits, one kernel
// per 8-bit pass.  `scratch` holds onesweepScratchWords(n, bits) words and is
// cleared here.  `err` receives bit 8 if a look-back wait gave up.
cudaError_t radixSortOnesweep(uint32_t* keys_a, uint32_t* vals_a, uint32_t* keys_b, uint32_t* vals_b, size_t n,
                              int bits, uint32_t* scratch, uint32_t* err, bool* result_in_b, cudaStream_t st) {
    *result_in_b = false;
    if (n == 0) return cudaSuccess;
    if (n > kCountMask) return cudaErrorInvalidValue;
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    const int ntiles = (int)radixTiles(n);
    uint32_t* ghist = scratch;
    uint32_t* counters = scratch + (size_t)passes * 256;
    uint32_t* status = counters + 32;
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * onesweepScratchWords(n, bits), st);
    if (e != cudaSuccess) return e;
    const int hblocks = (int)std::min<size_t>((n + kThreads * 16 - 1) / (kThreads * 16), 148 * 4);
    noteLaunches(1 + passes);
    onesweepHistKernel<<<hblocks, kThreads, 0, st>>>(keys_a, (uint32_t)n, passes, bits, ghist);
    uint32_t *kin = keys_a, *vin = vals_a, *kout = keys_b, *vout = vals_b;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        int pass_bits = bits - shift < 8 ? bits - shift : 8;
        if (pass_bits <= 0) pass_bits = 1;
        const uint32_t mask = (1u << pass_bits) - 1u;
        uint32_t* stat = status + (size_t)p * ntiles * 256;
        if (p == 0)
            onesweepPassKernel<true><<<ntiles, kThreads, 0, st>>>(kin, vin, kout, vout, (uint32_t)n, shift, mask,
                                                                  ghist + 256 * p, counters + p, stat, err);
        else
            onesweepPassKernel<false><<<ntiles, kThreads, 0, st>>>(kin, vin, kout, vout, (uint32_t)n, shift, mask,
                                                                   ghist + 256 * p, counters + p, stat, err);
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

}  // namespace mpm
