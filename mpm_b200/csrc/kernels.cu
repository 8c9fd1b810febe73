// kernels.cu -- the MPM step kernels for sm_100a.
//
//   keyKernel       cell keys of the live particle order (first step / after uploads)
//   compactOnesweepKernel   work items from per-block particle counts (P2G's,
//                   with their per-combination lists, and G2P's)
//   stressKernel    V0 * stress (tau) from Fe, Fp (first step / after uploads)
//   p2gKernel       deterministic block scatter by whole CTAs
//                   (src/mpm_solver3d.cu:237-294, src/apic_mpm_solver3d.cu:245-304)
//   p2gWarpKernel   the same scatter by single warps for small work items
//                   (bitwise p2gKernel's tiles)
//   gridKernel      tile merge + gravity + velocity update + collision in one
//                   pass (src/mpm_solver3d.cu:394-426, src/grid3d.cu:36-41)
//   g2pKernel       gather + transfer blend + Fe/Fp plasticity + SVD + next
//                   step's stress + particle collision + advection + next key
//                   (src/mpm_solver3d.cu:316-391,428-445; apic :326-388)
//   split-mode kernels for the reference's sub-step API.
#include <cuda.h>  // CUtensorMap and its enums (the encoder is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>

#include "engine_host.hpp"
#include "mpm_math.cuh"
#include "particle_common.cuh"

#include <atomic>
#include <cstdlib>

namespace mpm {

static std::atomic<uint64_t> g_launches{0};
void noteLaunches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t kernelLaunches() { return g_launches.load(std::memory_order_relaxed); }

namespace {


__device__ __forceinline__ float ldg(const float* p) { return __ldg(p); }

// Asynchronous 4-byte global -> shared copies (cp.async, L1-allocating).
__device__ __forceinline__ void cpAsync4(float* smem_dst, const float* gsrc) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cpAsyncWaitAll() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

constexpr int kPreStride = 19;  // odd: rows of consecutive threads fall in different banks


__device__ __forceinline__ uint32_t outsideKey(const SceneDev& sc) { return (sc.block_base + sc.nblocks) << 6; }

__device__ __forceinline__ uint32_t particleKey(const SceneDev& sc, const float* x, uint32_t* err) {
    int base[3];
    bool fin = isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]);
    if (!fin) atomicOr(err, ERR_NONFINITE);
    if (fin && stencilBase(sc, x, base)) return makeKey(sc, base);
    return outsideKey(sc);
}


// tau = V0 * (dPsi/dFe) Fe^T, symmetric (xx yy zz xy xz yz), from the SVD of Fe.
//  fixed corotated (src/material_point3d.cu:110-128):
//     2 mu (Fe - R) Fe^T + la (J-1) J I  =  2 mu U diag(s(s-1)) U^T + la (J-1) J I
//  Neo-Hookean (:131-155), with s clamped to >= FLT_EPSILON (Fe projected):
//     mu (Fe Fe^T - I) + la ln(J) I      =  mu U diag(s^2) U^T - mu I + la ln J I
__device__ __forceinline__ void tauFromSvd(int model, const float* U, const float* s, float mu, float la, float V0,
                                           float* tau) {
    float d[3], diag;
    float J = s[0] * s[1] * s[2];
    if (model == MPM_MODEL_NEO_HOOKEAN) {
#pragma unroll
        for (int k = 0; k < 3; ++k) d[k] = mu * s[k] * s[k];
        diag = la * logf(J) - mu;
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) d[k] = 2.0f * mu * s[k] * (s[k] - 1.0f);
        diag = la * (J - 1.0f) * J;
    }
    const int I[6] = {0, 1, 2, 0, 0, 1}, Jx[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
    for (int e = 0; e < 6; ++e) {
        int i = I[e], j = Jx[e];
        float v = U[3 * i] * d[0] * U[3 * j] + U[3 * i + 1] * d[1] * U[3 * j + 1] + U[3 * i + 2] * d[2] * U[3 * j + 2];
        if (e < 3) v += diag;
        tau[e] = V0 * v;
    }
}

// Stress of a particle from its current Fe (Neo-Hookean projects Fe in place).
__device__ __forceinline__ void stressFromFe(const MaterialDev& m, float* Fe, const float* Fp, float V0, float* tau) {
    float U[9], V[9], s[3];
    svd3(Fe, U, s, V);
    float mu, la;
    plasticLame(m, Fp, mu, la);
    if (m.model == MPM_MODEL_NEO_HOOKEAN) {
        bool proj = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            proj |= s[k] < kFltEps;
            s[k] = fmaxf(s[k], kFltEps);
        }
        if (proj) {
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    Fe[3 * i + j] = U[3 * i] * s[0] * V[3 * j] + U[3 * i + 1] * s[1] * V[3 * j + 1] +
                                    U[3 * i + 2] * s[2] * V[3 * j + 2];
        }
    }
    tauFromSvd(m.model, U, s, mu, la, V0, tau);
}

__device__ __forceinline__ int sceneOfBlock(const uint32_t* scene_block_base, int nscenes, uint32_t b) {
    int lo = 0, hi = nscenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (scene_block_base[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

}  // namespace

// ---------------------------------------------------------------------------
// Keys of the live particle order (used when keys were not produced by G2P).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) keyKernel(const SceneDev* __restrict__ scenes, int parity,
                                                       uint32_t* __restrict__ keys, uint32_t* __restrict__ block_count,
                                                       uint32_t* __restrict__ err) {
    const SceneDev& sc = scenes[blockIdx.y];
    const float* f = sc.buf[parity].f;
    const size_t cap = sc.cap;
    // whole warps iterate together, so that a warp's particles of one block
    // add to its count with one atomic (cell-sorted particles share blocks)
    const uint32_t n_round = (sc.n + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n_round; i += gridDim.x * kThreads) {
        const bool valid = i < sc.n;
        uint32_t blk = 0xffffffffu;
        if (valid) {
            float x[3] = {f[(F_X + 0) * cap + i], f[(F_X + 1) * cap + i], f[(F_X + 2) * cap + i]};
            const uint32_t key = particleKey(sc, x, err);
            keys[sc.key_offset + i] = key;
            blk = key >> 6;
        }
        const uint32_t peers = __match_any_sync(0xffffffffu, blk);
        if (valid && (int)(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&block_count[blk], (uint32_t)__popc(peers));
    }
}

// Block compaction in one kernel: each CTA scans a tile of 1024 block counts,
// publishes the tile's (work items, particles) sums and looks back over the
// earlier tiles' published words (single-pass scan, dynamic tile ids, every
// wait bounded), then writes the work items, slots and outside items of its
// blocks and clears their counts.  Word layout: [63:62] flag, [61:32] items,
// [31:0] particles.
constexpr int kCompactPer = 4;
constexpr int kCompactTile = kThreads * kCompactPer;
constexpr unsigned long long kCFlagAgg = 1ull << 62, kCFlagPrefix = 2ull << 62, kCFlagMask = 3ull << 62;

__device__ __forceinline__ unsigned long long blockExclusiveScanU64(unsigned long long x, unsigned long long* total) {
    __shared__ unsigned long long wt[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wt[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        unsigned long long t = lane < kWarps ? wt[lane] : 0ull, ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o) ti += y;
        }
        if (lane < kWarps) wt[lane] = ti - t;
        const unsigned long long tl = __shfl_sync(0xffffffffu, ti, kWarps - 1);
        if (lane == 0) *total = tl;
    }
    __syncthreads();
    const unsigned long long r = inc - x + wt[warp];
    __syncthreads();
    return r;
}

// The particles [start, start + count) of block b as `items` work items of
// nearly equal size: count / items each, the first count % items one more.
__device__ __forceinline__ void splitItems(BlockItem* out, uint32_t b, uint32_t start, uint32_t count,
                                           uint32_t items, uint32_t scene) {
    const uint32_t base = count / items, rem = count % items;
    uint32_t off = 0;
    for (uint32_t q = 0; q < items; ++q) {
        const uint32_t len = base + (q < rem ? 1u : 0u);
        out[q] = BlockItem{b, start + off, len, scene};
        off += len;
    }
}

__global__ void __launch_bounds__(kThreads) compactOnesweepKernel(
    uint32_t* __restrict__ block_count, uint32_t total_blocks, const uint32_t* __restrict__ scene_block_base,
    int nscenes, BlockItem* __restrict__ active, BlockItem* __restrict__ outside, uint32_t* __restrict__ counters,
    int32_t* __restrict__ block_slot, unsigned long long* __restrict__ status, uint32_t* __restrict__ tile_counter,
    uint32_t ntiles, uint32_t chunk, BlockItem* __restrict__ g2p_items, uint32_t g2p_cap, ComboSplit split,
    uint32_t* __restrict__ p2g_lists, uint32_t p2g_list_cap, const SceneDev* __restrict__ scenes,
    uint32_t* __restrict__ err) {
    __shared__ uint32_t tile_s;
    __shared__ unsigned long long tot, excl_s;
    if (threadIdx.x == 0) tile_s = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = tile_s;
    const uint32_t b0 = tile * kCompactTile + threadIdx.x * kCompactPer;
    unsigned long long packed[kCompactPer];
    unsigned long long sum = 0;
#pragma unroll
    for (int j = 0; j < kCompactPer; ++j) {
        const uint32_t b = b0 + j;
        unsigned long long v = 0;
        if (b < total_blocks) {
            const uint32_t c = block_count[b];
            const int s = sceneOfBlock(scene_block_base, nscenes, b);
            const bool out = (b == scene_block_base[s + 1] - 1);
            const unsigned long long items = (c > 0 && !out) ? (unsigned long long)((c + chunk - 1) / chunk) : 0ull;
            v = (items << 32) | (unsigned long long)c;
        }
        packed[j] = v;
        sum += v;
    }
    unsigned long long run = blockExclusiveScanU64(sum, &tot);
    if (threadIdx.x == 0) {
        unsigned long long excl = 0;
        if (tile == 0) {
            atomicExch(&status[0], kCFlagPrefix | tot);
        } else {
            atomicExch(&status[tile], kCFlagAgg | tot);
            // 8 predecessor words per round trip (independent loads)
            int t = (int)tile - 1;
            int polls = 0;
            bool done = false;
            while (!done && t >= 0) {
                unsigned long long w[8];
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    w[q] = (t - q >= 0) ? *(volatile const unsigned long long*)(status + (t - q)) : kCFlagPrefix;
                bool waiting = false;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    if (done || waiting) continue;
                    const unsigned long long f = w[q] & kCFlagMask;
                    if (f == 0) {  // not published yet: poll again from this tile
                        waiting = true;
                        continue;
                    }
                    excl += w[q] & ~kCFlagMask;
                    --t;
                    if (f == kCFlagPrefix) done = true;
                }
                if (waiting) {
                    if (++polls > (1 << 22)) {  // never expected: give up instead of hanging
                        atomicOr(err, 16u);
                        break;
                    }
                    __nanosleep(32);
                }
            }
            atomicExch(&status[tile], kCFlagPrefix | (excl + tot));
        }
        excl_s = excl;
        if (tile == ntiles - 1) counters[0] = (uint32_t)((excl + tot) >> 32);
    }
    __syncthreads();
    run += excl_s;
    // Slots of this thread's G2P items: one atomic per warp when every block
    // of the warp that has items belongs to one combination (the common
    // case), else one per block.
    int scn[kCompactPer];
    uint32_t gtot = 0;
    int gcombo = -1;
    bool mixed = false;
#pragma unroll
    for (int j = 0; j < kCompactPer; ++j) {
        const uint32_t b = b0 + j;
        scn[j] = 0;
        if (b >= total_blocks) continue;
        scn[j] = sceneOfBlock(scene_block_base, nscenes, b);
        if ((packed[j] >> 32) == 0) continue;
        const uint32_t count = (uint32_t)(packed[j] & 0xffffffffull);
        const int k = scenes[scn[j]].combo;
        gtot += (count + split.g2p_chunk[k] - 1) / split.g2p_chunk[k];
        if (gcombo < 0) gcombo = k;
        else mixed |= k != gcombo;
    }
    const int lane = threadIdx.x & 31;
    const unsigned has = __ballot_sync(0xffffffffu, gtot > 0);
    const int lead = __shfl_sync(0xffffffffu, gcombo, has ? __ffs(has) - 1 : 0);
    const bool warp_fast = __all_sync(0xffffffffu, gtot == 0 || (!mixed && gcombo == lead));
    uint32_t gnext = 0;
    if (warp_fast && has) {
        uint32_t inc = gtot;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        uint32_t base = 0;
        if (lane == 31) base = atomicAdd(&counters[kG2PCountWord + lead], inc);
        gnext = __shfl_sync(0xffffffffu, base, 31) + inc - gtot;
    }
    // Slots of this thread's P2G items in their combination's lists: list 0
    // for items of at most the combination's warp threshold (P2G by warps),
    // list 1 for the others -- those of at least kBigItem particles from its
    // front, the rest from its back (class 2); aggregated per warp like the
    // G2P items.  The items of at most kWarpAutoMax particles are counted
    // as well (class 3).
    uint32_t pnext[3] = {0u, 0u, 0u};
    if (p2g_lists && warp_fast && has) {
        uint32_t ptot[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int j = 0; j < kCompactPer; ++j) {
            const uint32_t items = (uint32_t)(packed[j] >> 32);
            if (b0 + j >= total_blocks || !items) continue;
            const uint32_t size = ((uint32_t)(packed[j] & 0xffffffffull) + items - 1) / items;
            ptot[size <= split.p2g_warp_max[lead] ? 0 : (size >= kBigItem ? 1 : 2)] += items;
            if (size <= kWarpAutoMax) ptot[3] += items;
        }
        const int words[4] = {kP2GListWord + 2 * lead, kP2GListWord + 2 * lead + 1, kP2GBackWord + lead,
                              kP2GSmallWord + lead};
#pragma unroll
        for (int cls = 0; cls < 4; ++cls) {
            uint32_t inc = ptot[cls];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += y;
            }
            uint32_t base = 0;
            if (lane == 31 && inc) base = atomicAdd(&counters[words[cls]], inc);
            if (cls < 3) pnext[cls] = __shfl_sync(0xffffffffu, base, 31) + inc - ptot[cls];
        }
    }
#pragma unroll
    for (int j = 0; j < kCompactPer; ++j) {
        const uint32_t b = b0 + j;
        if (b >= total_blocks) break;
        const unsigned long long v = packed[j];
        const uint32_t count = (uint32_t)(v & 0xffffffffull);
        const uint32_t items = (uint32_t)(v >> 32);
        const uint32_t start = (uint32_t)(run & 0xffffffffull);
        const int scene = scn[j];
        // a block's items have count / items particles, the first
        // count % items of them one more (sizes differ by at most one)
        if (items) {
            const uint32_t slot = (uint32_t)(run >> 32);
            splitItems(active + slot, b, start, count, items, (uint32_t)scene);
            block_slot[b] = (int32_t)slot;
            // G2P's items of the block, in its combination's list at slots
            // taken from a counter (their order does not matter)
            const int k = scenes[scene].combo;
            const uint32_t parts = (count + split.g2p_chunk[k] - 1) / split.g2p_chunk[k];
            uint32_t g0;
            if (warp_fast) {
                g0 = gnext;
                gnext += parts;
            } else {
                g0 = atomicAdd(&counters[kG2PCountWord + k], parts);
            }
            splitItems(g2p_items + (size_t)k * g2p_cap + g0, b, start, count, parts, (uint32_t)scene);
            if (p2g_lists) {
                const uint32_t size = (count + items - 1) / items;
                const int cls = size <= split.p2g_warp_max[k] ? 0 : (size >= kBigItem ? 1 : 2);
                const int words[3] = {kP2GListWord + 2 * k, kP2GListWord + 2 * k + 1, kP2GBackWord + k};
                uint32_t p0;
                if (warp_fast) {
                    p0 = pnext[cls];
                    pnext[cls] += items;
                } else {
                    p0 = atomicAdd(&counters[words[cls]], items);
                    if (size <= kWarpAutoMax) atomicAdd(&counters[kP2GSmallWord + k], items);
                }
                uint32_t* lst = p2g_lists + (size_t)(2 * k + (cls == 0 ? 0 : 1)) * p2g_list_cap;
                for (uint32_t q = 0; q < items; ++q) {
                    if (cls == 2) lst[p2g_list_cap - 1 - (p0 + q)] = slot + q;  // from the back
                    else lst[p0 + q] = slot + q;
                }
            }
        } else {
            block_slot[b] = -1;
            if (count > 0) {
                const uint32_t nitems = (count + chunk - 1) / chunk;
                const uint32_t o = atomicAdd(&counters[1], nitems);
                splitItems(outside + o, b, start, count, nitems, (uint32_t)scene);
            }
        }
        block_count[b] = 0;
        run += v;
    }
}

// ---------------------------------------------------------------------------
// tau from Fe/Fp for the live order (first step, after uploads).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads) stressKernel(const SceneDev* __restrict__ scenes, int parity) {
    const SceneDev& sc = scenes[blockIdx.y];
    float* f = sc.buf[parity].f;
    const uint16_t* mat = sc.buf[parity].mat;
    const size_t cap = sc.cap;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads) {
        float Fe[9], Fp[9], tau[6];
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            Fe[k] = f[(F_FE + k) * cap + i];
            Fp[k] = f[(F_FP + k) * cap + i];
        }
        // Fe = I (a new scene): tau = 0 exactly for both models (R = I,
        // J = 1), without the FP32 SVD's round-off in s (~1e-7), which a
        // stiff material turns into a spurious force at light surface nodes.
        bool identity = true;
#pragma unroll
        for (int k = 0; k < 9; ++k) identity = identity && Fe[k] == ((k % 4 == 0) ? 1.f : 0.f);
        if (identity) {
#pragma unroll
            for (int k = 0; k < 6; ++k) f[(F_TAU + k) * cap + i] = 0.f;
            continue;
        }
        MaterialDev m = sc.mats[sc.nmat > 1 ? mat[i] : 0];
        stressFromFe(m, Fe, Fp, f[F_VOL * cap + i], tau);
        if (m.model == MPM_MODEL_NEO_HOOKEAN)
#pragma unroll
            for (int k = 0; k < 9; ++k) f[(F_FE + k) * cap + i] = Fe[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) f[(F_TAU + k) * cap + i] = tau[k];
    }
}

// ---------------------------------------------------------------------------
// P2G: one CTA per active 4^3-cell block (persistent loop).  Each warp takes
// whole cells (dynamically, cell by cell); its lanes own the S^3 stencil
// nodes of the cell and accumulate the cell's particles, in sorted order, in
// registers.  Cell partial sums are merged into the (S+3)^3 block tile by a
// fixed-order gather, and the tile is written to scratch.  Which warp takes a
// cell does not matter: every sum has a fixed order, no floating-point
// atomics, bitwise deterministic.
//
// Staged payload of a particle (floats, 16-byte aligned rows):
//   shared part (one broadcast float4 per 4 values)
//     APIC / SPLIT : m, q[3] | hC[0..3] | hC[4..7] | hC[8], T[0..2] | T[3..5], -
//                    q = m v - m C delta, hC = h m C (C = B D^-1), T = stress term
//     PIC-FLIP     : m, m v[3] | T[0..3] | T[4..5], -, -
//     MASS         : m, -, -, -
//   weights: (N(d), N'(d)/h) pairs per axis and stencil offset (float2)
// ---------------------------------------------------------------------------
// Staging-record stride (floats): a multiple of 4 (float4 loads) whose
// multiples q * P, q < groups, start at least 4 banks apart, so that the
// broadcast loads of a warp's particle groups never share a bank.
__host__ __device__ constexpr bool stageStrideOk(int P, int groups) {
    for (int a = 0; a < groups; ++a)
        for (int b = a + 1; b < groups; ++b) {
            const int d = ((b - a) * P) % 32;
            if (d < 4 || d > 28) return false;
        }
    return true;
}
__host__ __device__ constexpr int stageStride(int base, int groups) {
    int P = (base + 3) / 4 * 4;
    while (!stageStrideOk(P, groups)) P += 4;
    return P;
}

// One lane's sums for one stencil node, in packed FP32 pairs so that the
// x and y components go through one __ffma2_rn (two exactly rounded FMAs: the
// same results as fmaf), and the mass with the z momentum:
//   mz = (m, p_z), pxy = (p_x, p_y), fxy = (f_x, f_y), fz = f_z.
// Field f of the tile layout (m, p[3], f[3]) is get(f).
struct NodeAcc {
    float2 mz, pxy, fxy;
    float fz;
    __device__ __forceinline__ void zero() {
        mz = pxy = fxy = make_float2(0.f, 0.f);
        fz = 0.f;
    }
    __device__ __forceinline__ float get(int f) const {
        return f == 0 ? mz.x : f == 1 ? pxy.x : f == 2 ? pxy.y : f == 3 ? mz.y : f == 4 ? fxy.x : f == 5 ? fxy.y : fz;
    }
};

template <int S, int MODE, int STAGE = 16>
struct P2GLayout {
    static constexpr int F = modeFields(MODE);
    static constexpr int NS = S * S * S;              // stencil nodes
    static constexpr int PAIRS = S * S;               // (a, b) columns; a lane owns one column of S nodes
    static constexpr int G = 32 / PAIRS;              // particle groups per warp (one particle each per pass)
    static constexpr int TN = tileNodes(S);
    static constexpr int SH = (MODE == MODE_MASS) ? 4 : (MODE == MODE_FLIP ? 12 : 20);  // shared floats
    static constexpr int WB = SH;                     // weight pairs start
    static constexpr int P = stageStride(SH + 6 * S, G);
    static constexpr int kStage = STAGE;              // particles staged per warp round
    static constexpr int kSlots = 32;                 // segment partials per round (<= 32: one per lane)
    static constexpr int kSeg = 96;                   // particles per segment (at most)
    static constexpr int kMaxSeg = 128;               // >= 64 + kBlockChunk / kSeg + 1
    static constexpr int kCtlInts = 2 * 64 + 3 * kMaxSeg + 4;
    // dynamic shared memory of nw warps: stage [nw][kStage][P] floats,
    // partials [kSlots][F][NS] floats, then the control ints (cellBeg[64],
    // cellEnd[64], segCell/segBeg/segEnd[kMaxSeg], ctl[4]); the kernel takes
    // its pointers from these offsets
    static constexpr size_t smemFor(int nw) {
        return ((size_t)nw * kStage * P + (size_t)kSlots * F * NS) * 4 + (size_t)kCtlInts * 4;
    }
    // Threads per CTA.  Dense cubic scenes (staging 24 or 32 particles per
    // pass) get two CTAs of 12 warps per SM where they fit its shared memory
    // (at most ~113 KB each): 24 warps, the register file's limit at 80
    // registers, working on two blocks.  Otherwise CTAs of 8 warps, three per
    // SM where they fit: sparse scenes (staging 16, chosen below 8 particles
    // per cell) have too few staging windows per block to keep 12 warps busy
    // (8.4M-particle slab P2G 2.8 ms with 8 warps against 3.4 ms with 12).
    static constexpr int NT = (S == 4 && STAGE >= 24 && smemFor(12) <= 113 * 1024) ? 384 : 256;
    static constexpr int NW = NT / 32;
    // CTAs per SM the launch bound asks for: as many as the shared memory
    // holds (228 KB per SM, 1 KB of it reserved per CTA), at most 3 (80
    // registers); the register budget follows from it.
    static constexpr int MIN_CTAS = NT == 384 ? 2 : ((smemFor(8) + 1024) * 3 <= 228 * 1024 ? 3 : 2);
    static constexpr int TJ = (TN + NT - 1) / NT;
    static constexpr size_t kPartialOff = (size_t)NW * kStage * P;
    static constexpr size_t kCtlOff = kPartialOff + (size_t)kSlots * F * NS;
    static constexpr size_t smemBytes = smemFor(NW);
    static_assert(smemBytes == kCtlOff * 4 + (size_t)kCtlInts * 4, "layout");
    static_assert(kMaxSeg >= 64 + (int)(kBlockChunk / kSeg) + 1, "segment list too small");
};

// P2G staging of one particle (sorted position gs) at `my`: mass, momentum
// terms, stress factors and stencil weights in the layout of P2GStage.  The
// CTA and warp P2G kernels share it (and p2gAccumulate), so their sums are
// bitwise the same.
template <int S, int MODE, int P, int WB>
__device__ __forceinline__ void p2gStageParticle(const StepArgs& args, const SceneDev& sc, const float* pf, size_t cap,
                                                 float dt, float h, float inv_h, uint32_t gs, float* my) {
    uint32_t old = args.perm[gs] - sc.key_offset;
    const bool bad = old >= sc.n;  // range check: flag and contribute nothing
    if (bad) {
        atomicOr(args.err, ERR_INDEX);
        old = 0;
    }
    float x[3] = {ldg(pf + (F_X + 0) * cap + old), ldg(pf + (F_X + 1) * cap + old),
                  ldg(pf + (F_X + 2) * cap + old)};
    int base[3];
    stencilBase(sc, x, base);
    float delta[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float gp0 = __fadd_rn(sc.origin[a], __fmul_rn(h, (float)base[a]));
        delta[a] = x[a] - gp0;
        // Node distances.  The linear kernel's weights
        // have relative error ~ulp(d)/w near |d| = 1, so it
        // forms each one as the reference does,
        // (x_p - (o + h i)) / h; the B-splines are smooth
        // there and use d0 - k (exact subtraction).
        float dk[S], wk[S], dwk[S];
        if (S == 2) {
#pragma unroll
            for (int k = 0; k < S; ++k) {
                const float gp = __fadd_rn(sc.origin[a], __fmul_rn(h, (float)(base[a] + k)));
                dk[k] = __fdiv_rn(__fsub_rn(x[a], gp), h);
            }
        } else {
            dk[0] = __fdiv_rn(delta[a], h);
#pragma unroll
            for (int k = 1; k < S; ++k) dk[k] = dk[0] - (float)k;
        }
        splineWeights<S>(dk, wk, dwk);
#pragma unroll
        for (int k = 0; k < S; ++k) {
            if (MODE == MODE_MASS) {
                my[WB + a * S + k] = wk[k];
            } else {  // (w, w'/h) pairs: 8-byte stores (WB is even, rows 16-byte aligned)
                *reinterpret_cast<float2*>(my + WB + 2 * (a * S + k)) = make_float2(wk[k], dwk[k] * inv_h);
            }
        }
    }
    const float m = bad ? 0.f : ldg(pf + F_MASS * cap + old);
    if (MODE == MODE_MASS) my[0] = m;
    if (MODE != MODE_MASS) {
        float v[3] = {ldg(pf + (F_V + 0) * cap + old), ldg(pf + (F_V + 1) * cap + old),
                      ldg(pf + (F_V + 2) * cap + old)};
        const float ts = bad ? 0.f : ((MODE == MODE_APIC_FUSED) ? -dt : -1.0f);
        float T[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) T[k] = ts * ldg(pf + (F_TAU + k) * cap + old);
        // the row's header in 16-byte stores: (m, p), then the stress
        // factors (and APIC's h m C): the layout the accumulation reads
        float4* my4 = reinterpret_cast<float4*>(my);
        if (MODE == MODE_FLIP) {
            my4[0] = make_float4(m, m * v[0], m * v[1], m * v[2]);
            my4[1] = make_float4(T[0], T[1], T[2], T[3]);
            *reinterpret_cast<float2*>(my + 8) = make_float2(T[4], T[5]);
        } else {
            float mC[9];
            if (sc.transfer == MPM_TRANSFER_APIC) {
                const float md = m * sc.dinv;
#pragma unroll
                for (int k = 0; k < 9; ++k) mC[k] = md * ldg(pf + (F_B + k) * cap + old);
            } else {
#pragma unroll
                for (int k = 0; k < 9; ++k) mC[k] = 0.f;
            }
            float q[3], hC[9];
#pragma unroll
            for (int a = 0; a < 3; ++a)
                q[a] = m * v[a] - (mC[3 * a] * delta[0] + mC[3 * a + 1] * delta[1] + mC[3 * a + 2] * delta[2]);
#pragma unroll
            for (int k = 0; k < 9; ++k) hC[k] = h * mC[k];
            my4[0] = make_float4(m, q[0], q[1], q[2]);
            my4[1] = make_float4(hC[0], hC[1], hC[2], hC[3]);
            my4[2] = make_float4(hC[4], hC[5], hC[6], hC[7]);
            my4[3] = make_float4(hC[8], T[0], T[1], T[2]);
            my4[4] = make_float4(T[3], T[4], T[5], 0.f);  // [19] is padding of the header
        }
    }
}

// One lane's sums over the staged particles q0, q0 + G, ... below qhi (its
// group's share of a segment, in order) for the stencil column (na, nb).
template <int S, int MODE, int P, int WB, int G>
__device__ __forceinline__ void p2gAccumulate(const float* st, int q0, int qhi, int na, int nb, NodeAcc* acc) {
    const float fa = (float)na, fb = (float)nb;
    for (int q = q0; q < qhi; q += G) {
        const float* pq = st + q * P;
        const float4 s0 = *reinterpret_cast<const float4*>(pq);
        const float m = s0.x;
        if (MODE == MODE_MASS) {
            const float mw = m * (pq[WB + na] * pq[WB + S + nb]);
#pragma unroll
            for (int c = 0; c < S; ++c) acc[c].mz.x = fmaf(mw, pq[WB + 2 * S + c], acc[c].mz.x);
            continue;
        }
        // column factors: w = wab Z_c and
        // T grad w = Z_c A + Z'_c Bz with A = T (X'Y, XY', 0), Bz = T (0, 0, XY)
        const float2 xa = *reinterpret_cast<const float2*>(pq + WB + 2 * na);
        const float2 yb = *reinterpret_cast<const float2*>(pq + WB + 2 * (S + nb));
        const float wab = xa.x * yb.x, dab = xa.y * yb.x, adb = xa.x * yb.y;
        float T[6];
        float2 uxy, mu;  // (u_x, u_y) and (m, u_z)
        float2 hxy = make_float2(0.f, 0.f);
        float hz = 0.f;
        if (MODE == MODE_FLIP) {
            const float4 s1 = *reinterpret_cast<const float4*>(pq + 4);
            const float4 s2 = *reinterpret_cast<const float4*>(pq + 8);
            T[0] = s1.x; T[1] = s1.y; T[2] = s1.z; T[3] = s1.w; T[4] = s2.x; T[5] = s2.y;
            uxy = make_float2(s0.y, s0.z);
            mu = make_float2(m, s0.w);
        } else {
            const float4 s1 = *reinterpret_cast<const float4*>(pq + 4);
            const float4 s2 = *reinterpret_cast<const float4*>(pq + 8);
            const float4 s3 = *reinterpret_cast<const float4*>(pq + 12);
            const float4 s4 = *reinterpret_cast<const float4*>(pq + 16);
            const float hC[9] = {s1.x, s1.y, s1.z, s1.w, s2.x, s2.y, s2.z, s2.w, s3.x};
            T[0] = s3.y; T[1] = s3.z; T[2] = s3.w; T[3] = s4.x; T[4] = s4.y; T[5] = s4.z;
            const float qv[3] = {s0.y, s0.z, s0.w};
            float u[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) u[i] = fmaf(hC[3 * i], fa, fmaf(hC[3 * i + 1], fb, qv[i]));
            uxy = make_float2(u[0], u[1]);
            mu = make_float2(m, u[2]);
            hxy = make_float2(hC[2], hC[5]);
            hz = hC[8];
        }
        const float2 Axy = make_float2(fmaf(T[0], dab, T[3] * adb), fmaf(T[3], dab, T[1] * adb));
        const float Az = fmaf(T[4], dab, T[5] * adb);
        const float2 Bxy = make_float2(T[4] * wab, T[5] * wab);
        const float Bz = T[2] * wab;
#pragma unroll
        for (int c = 0; c < S; ++c) {
            const float2 zc = *reinterpret_cast<const float2*>(pq + WB + 2 * (2 * S + c));
            const float wgt = wab * zc.x;
            const float2 w2 = make_float2(wgt, wgt), zx2 = make_float2(zc.x, zc.x),
                         zy2 = make_float2(zc.y, zc.y);
            if (c > 0 && MODE != MODE_FLIP) {  // u at node c: u += h C e_z, component-wise
                uxy = __fadd2_rn(uxy, hxy);
                mu.y += hz;
            }
            // m += m w and p_z += w u_z in one pair
            acc[c].mz = __ffma2_rn(mu, w2, acc[c].mz);
            if (MODE == MODE_APIC_FUSED) {
                // p += w u + Z_c A + Z'_c Bz (the order of the nested fmaf)
                acc[c].pxy = __ffma2_rn(zy2, Bxy, __ffma2_rn(zx2, Axy, __ffma2_rn(w2, uxy, acc[c].pxy)));
                acc[c].mz.y = fmaf(zc.y, Bz, fmaf(zc.x, Az, acc[c].mz.y));
            } else {  // PIC-FLIP and SPLIT keep p and f apart
                acc[c].pxy = __ffma2_rn(w2, uxy, acc[c].pxy);
                acc[c].fxy = __ffma2_rn(zy2, Bxy, __ffma2_rn(zx2, Axy, acc[c].fxy));
                acc[c].fz = fmaf(zc.y, Bz, fmaf(zc.x, Az, acc[c].fz));
            }
        }
    }
}

template <int S, int MODE, int STAGE>
__global__ void __launch_bounds__(P2GLayout<S, MODE, STAGE>::NT, P2GLayout<S, MODE, STAGE>::MIN_CTAS)
    p2gKernel(StepArgs args, int want_transfer) {
    using L = P2GLayout<S, MODE, STAGE>;
    constexpr int F = L::F;
    extern __shared__ float4 smem4[];
    float* smem = reinterpret_cast<float*>(smem4);
    float* stage = smem;                     // [warp][kStage][P]
    float* partial = smem + L::kPartialOff;  // [slot][F][NS]
    int* cellBeg = (int*)(smem + L::kCtlOff);
    int* cellEnd = cellBeg + 64;
    int* segCell = cellEnd + 64;                                // segment list, in cell order
    int* segBeg = segCell + L::kMaxSeg;
    int* segEnd = segBeg + L::kMaxSeg;
    int* ctl = segEnd + L::kMaxSeg;                             // [0] segments, [1] next segment

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // lane -> particle group grp and stencil column (na, nb): the lane
    // accumulates nodes (na, nb, 0..S-1) for the group's particles
    // grp, grp + G, grp + 2G, ... of each staged batch.
    const int grp = lane / L::PAIRS, na = (lane % L::PAIRS) % S, nb = (lane % L::PAIRS) / S;
    const bool lane_on = grp < L::G;
    // the combination's list of items for whole CTAs, or every active item
    const uint32_t* list = args.p2g_lists ? args.p2g_lists + (size_t)(2 * args.combo + 1) * args.p2g_list_cap : nullptr;
    // the long items from the list's front first, then the others from its
    // back, then -- unless the warp kernel takes them -- the small items
    const uint32_t nfront = list ? args.counters[kP2GListWord + 2 * args.combo + 1] : 0u;
    const uint32_t nlist1 = list ? nfront + args.counters[kP2GBackWord + args.combo] : 0u;
    const uint32_t nsmall = list ? args.counters[kP2GListWord + 2 * args.combo] : 0u;
    const uint32_t nwork = !list ? args.counters[0]
                                 : nlist1 + (p2gWarpTakesSmall(args.p2g_warp, nsmall) ? 0u : nsmall);
    const uint32_t* small = list ? args.p2g_lists + (size_t)(2 * args.combo) * args.p2g_list_cap : nullptr;
    spanBegin(args.spans, SPAN_P2G);
    __shared__ uint32_t item_s;
    __shared__ SceneDev sc_s;
    for (;;) {
        const uint32_t wi = nextWorkItem(args.sched, nwork, &item_s);
        if (wi >= nwork) break;
        const uint32_t w = !list ? wi
                           : wi < nfront ? list[wi]
                           : wi < nlist1 ? list[args.p2g_list_cap - 1 - (wi - nfront)]
                                         : small[wi - nlist1];
        const BlockItem it = args.active[w];
        {
            const SceneDev& scg = args.scenes[it.scene];
            if (scg.S != S || (want_transfer >= 0 && scg.transfer != want_transfer)) continue;
            if (MODE == MODE_MASS && !scg.init_pass) continue;
        }
        // the scene's entry into shared memory: the staging reads its fields
        // per particle
        if (warp == 0) {
            const int4* src = reinterpret_cast<const int4*>(args.scenes + it.scene);
            int4* dst = reinterpret_cast<int4*>(&sc_s);
            for (int q = lane; q < (int)(sizeof(SceneDev) / 16); q += 32) dst[q] = src[q];
        }
        for (int c = threadIdx.x; c < 64; c += L::NT) cellBeg[c] = cellEnd[c] = 0;
        __syncthreads();
        const SceneDev& sc = sc_s;
        const float* pf = sc.buf[args.parity].f;
        const size_t cap = sc.cap;
        const uint32_t i0 = it.start, icount = it.count;

        // Cell ranges inside the work item (keys are sorted by cell).
        for (uint32_t i = threadIdx.x; i < icount; i += L::NT) {
            uint32_t g = i0 + i;
            uint32_t c = args.sorted_keys[g] & 63u;
            if (i == 0 || (args.sorted_keys[g - 1] & 63u) != c) cellBeg[c] = (int)i;
            if (i == icount - 1 || (args.sorted_keys[g + 1] & 63u) != c) cellEnd[c] = (int)i + 1;
        }
        __syncthreads();
        // Segment list: every non-empty cell cut into runs of at most kSeg
        // particles, in cell order (warp 0; lane l owns cells 2l and 2l+1).
        if (warp == 0) {
            const int c0 = 2 * lane, c1 = 2 * lane + 1;
            const int b0 = cellBeg[c0], e0 = cellEnd[c0], b1 = cellBeg[c1], e1 = cellEnd[c1];
            const int n0 = e0 > b0 ? (e0 - b0 + L::kSeg - 1) / L::kSeg : 0;
            const int n1 = e1 > b1 ? (e1 - b1 + L::kSeg - 1) / L::kSeg : 0;
            int x = n0 + n1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            int off = x - (n0 + n1);
            for (int j = 0; j < n0; ++j, ++off) {
                segCell[off] = c0;
                segBeg[off] = b0 + j * L::kSeg;
                segEnd[off] = min(e0, b0 + (j + 1) * L::kSeg);
            }
            for (int j = 0; j < n1; ++j, ++off) {
                segCell[off] = c1;
                segBeg[off] = b1 + j * L::kSeg;
                segEnd[off] = min(e1, b1 + (j + 1) * L::kSeg);
            }
            if (lane == 31) {
                ctl[0] = x;
                ctl[1] = 0;
            }
        }
        __syncthreads();
        const int nseg = ctl[0];

        float tacc[L::TJ][F];
#pragma unroll
        for (int j = 0; j < L::TJ; ++j)
#pragma unroll
            for (int f = 0; f < F; ++f) tacc[j][f] = 0.f;

        const float dt = sc.dt, h = sc.h, inv_h = sc.inv_h;
        for (int r0 = 0; r0 < nseg; r0 += L::kSlots) {
            const int rend = min(nseg, r0 + L::kSlots);
            // ---- particle phase: warps take segments of this round dynamically ----
            float* st = stage + (size_t)warp * L::kStage * L::P;
            // The round's particles [rb, re) are cut into windows of kStage; a
            // warp takes a window and handles the segments that start in it:
            // several sparse cells share one staging pass, a long segment
            // takes several.  Each segment is summed by one warp, in order.
            const int rb = segBeg[r0], re = segEnd[rend - 1];
            const int nwin = (re - rb + L::kStage - 1) / L::kStage;
            while (true) {
                int wi = 0;
                if (lane == 0) wi = atomicAdd(&ctl[1], 1);
                wi = __shfl_sync(0xffffffffu, wi, 0);
                if (wi >= nwin) break;
                const int sl = r0 + lane;  // a round has at most 32 segments: one per lane
                const bool starts = sl < rend && (segBeg[sl] - rb) / L::kStage == wi;
                const unsigned own = __ballot_sync(0xffffffffu, starts);
                if (!own) continue;
                const int s_first = r0 + __ffs(own) - 1, s_last = r0 + 31 - __clz(own);
                const int cb = segBeg[s_first], ce = segEnd[s_last];
                int cur = s_first;  // segment being summed
                NodeAcc acc[S];
#pragma unroll
                for (int c = 0; c < S; ++c) acc[c].zero();
                for (int g0 = cb; g0 < ce; g0 += L::kStage) {
                    const int np = min(L::kStage, ce - g0);
                    if (lane < np) {
                        p2gStageParticle<S, MODE, L::P, L::WB>(args, sc, pf, cap, dt, h, inv_h,
                                                               i0 + (uint32_t)(g0 + lane), st + lane * L::P);
                    }
                    __syncwarp();
                    // the segments overlapping this pass, in order
                    while (cur <= s_last) {
                    const int se = segEnd[cur];
                    const int qlo = max(segBeg[cur], g0) - g0, qhi = min(se, g0 + np) - g0;
                    // group grp sums the segment's particles j = grp (mod G), in
                    // order, however the segment is cut into staging passes
                    const int jlo = g0 + qlo - segBeg[cur];
                    if (lane_on)
                        p2gAccumulate<S, MODE, L::P, L::WB, L::G>(st, qlo + (grp - jlo % L::G + L::G) % L::G, qhi, na,
                                                                  nb, acc);
                    if (se > g0 + np) break;  // the segment continues in the next pass
                    // Segment done: sum the groups' columns in group order into
                    // group 0 (fixed order, so the partial does not depend on
                    // timing), write its slot, start the next segment.
#pragma unroll
                    for (int c = 0; c < S; ++c) {
#pragma unroll
                        for (int f = 0; f < F; ++f) {
                            const float mine = acc[c].get(f);
                            float sum = mine;
#pragma unroll
                            for (int g = 1; g < L::G; ++g)
                                sum += __shfl_sync(0xffffffffu, mine, min(lane + g * L::PAIRS, 31));
                            if (grp == 0)
                                partial[(size_t)(cur - r0) * F * L::NS + f * L::NS + na + S * nb + L::PAIRS * c] = sum;
                        }
                        acc[c].zero();
                    }
                    ++cur;
                    }
                    __syncwarp();
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) ctl[1] = 0;  // next round's dynamic counter (no warp reads it until the barrier below)
            // ---- gather phase: fixed-order merge of this round's segments ----
#pragma unroll
            for (int j = 0; j < L::TJ; ++j) {
                const int tn = threadIdx.x + j * L::NT;
                if (tn < L::TN) {
                    const int tx = tn % (S + 3), ty = (tn / (S + 3)) % (S + 3), tz = tn / ((S + 3) * (S + 3));
                    for (int sg = r0; sg < rend; ++sg) {
                        const int cell = segCell[sg];
                        const int dx = tx - (cell & 3), dy = ty - ((cell >> 2) & 3), dz = tz - (cell >> 4);
                        if ((unsigned)dx >= (unsigned)S || (unsigned)dy >= (unsigned)S || (unsigned)dz >= (unsigned)S)
                            continue;
                        // stencil node index of the lane layout: a + S (b + S c)
                        const float* pc = partial + (size_t)(sg - r0) * F * L::NS + dx + S * (dy + S * dz);
#pragma unroll
                        for (int f = 0; f < F; ++f) tacc[j][f] += pc[f * L::NS];
                    }
                }
            }
            __syncthreads();
        }
        float* tile = args.tiles + (size_t)w * args.tile_stride;
#pragma unroll
        for (int j = 0; j < L::TJ; ++j) {
            const int tn = threadIdx.x + j * L::NT;
            if (tn < L::TN)
#pragma unroll
                for (int f = 0; f < F; ++f) tile[f * L::TN + tn] = tacc[j][f];
        }
    }
    spanEnd(args.spans, SPAN_P2G);
}


// ---------------------------------------------------------------------------
// P2G by whole warps for the small items (the combination's warp list).  Each
// warp takes an item and sums its particles segment by segment as p2gKernel
// does -- cells in order, each cut into segments of at most kSeg particles; a
// segment's particles summed per group in order, the groups then in lane
// order (p2gStageParticle, p2gAccumulate) -- and adds each segment's sums
// into its own shared-memory tile in segment order, the order of p2gKernel's
// merge: the tile is bitwise p2gKernel's, so which kernel takes an item
// changes no result.  No CTA barrier: an item of a few particles per cell
// spends most of p2gKernel's time in its per-item set-up, barriers and merge
// rounds.
// ---------------------------------------------------------------------------
template <int S, int MODE>
struct P2GWarpLayout {
    using D = P2GLayout<S, MODE, 16>;  // staging layout, column map and segment length
    static constexpr int F = D::F, TN = D::TN, P = D::P, WB = D::WB, G = D::G, PAIRS = D::PAIRS;
    static constexpr int kSeg = D::kSeg;
    static constexpr int kStage = 16;  // particles staged per pass
    static constexpr int NT = 256, NW = NT / 32;
    // per warp: its item's scene entry, its tile [F][TN], its staging rows
    // (field-major: a column's 16 lanes add to 16 different banks; a
    // node-major tile of 16-byte words had bank conflicts and was slower)
    static constexpr int kSceneFloats = (int)((sizeof(SceneDev) + 15) / 16 * 4);
    static constexpr int kTileFloats = (F * TN + 3) / 4 * 4;
    static constexpr int kWarpFloats = kSceneFloats + kTileFloats + kStage * P;
    static constexpr size_t smemBytes = (size_t)NW * kWarpFloats * 4;
    static constexpr int MIN_CTAS = (smemBytes + 1024) * 3 <= 228 * 1024 ? 3 : 2;
};

template <int S, int MODE>
__global__ void __launch_bounds__(P2GWarpLayout<S, MODE>::NT, P2GWarpLayout<S, MODE>::MIN_CTAS)
    p2gWarpKernel(StepArgs args) {
    using W = P2GWarpLayout<S, MODE>;
    constexpr int F = W::F, T = S + 3, TN = W::TN, G = W::G, PAIRS = W::PAIRS;
    extern __shared__ float4 smem4[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float* wbase = reinterpret_cast<float*>(smem4) + (size_t)warp * W::kWarpFloats;
    SceneDev& sc = *reinterpret_cast<SceneDev*>(wbase);
    float* tile = wbase + W::kSceneFloats;
    float* st = tile + W::kTileFloats;
    const int grp = lane / PAIRS, na = (lane % PAIRS) % S, nb = (lane % PAIRS) / S;
    const bool lane_on = grp < G;
    const uint32_t* list = args.p2g_lists + (size_t)(2 * args.combo) * args.p2g_list_cap;
    const uint32_t nwork = args.counters[kP2GListWord + 2 * args.combo];
    // the warps' item scheduler: [0] hands out list indices, [1] counts the
    // warps that have run out; the last of them clears both
    uint32_t* sched = args.sched + 2;
    const uint32_t warps = gridDim.x * (uint32_t)W::NW;
    // nothing for warps (the scheduler is untouched): p2gKernel takes the
    // small items when the list is too short to fill the GPU with warps
    if (nwork == 0 || !p2gWarpTakesSmall(args.p2g_warp, nwork)) return;
    NodeAcc acc[S];
    // a segment done: the groups' columns summed in group order (as
    // p2gKernel), added by group 0 into the tile nodes of the segment's cell
    auto finish = [&](int cell) {
        const int cx = cell & 3, cy = (cell >> 2) & 3, cz = cell >> 4;
#pragma unroll
        for (int c = 0; c < S; ++c) {
#pragma unroll
            for (int f = 0; f < F; ++f) {
                const float mine = acc[c].get(f);
                float sum = mine;
#pragma unroll
                for (int g = 1; g < G; ++g) sum += __shfl_sync(0xffffffffu, mine, min(lane + g * PAIRS, 31));
                if (grp == 0) tile[f * TN + (na + cx) + T * ((nb + cy) + T * (c + cz))] += sum;
            }
            acc[c].zero();
        }
        __syncwarp();  // the next segment's sums may land on the same nodes from other lanes
    };
    spanBegin(args.spans, SPAN_P2G);
    for (;;) {
        uint32_t wi = 0;
        if (lane == 0) {
            wi = atomicAdd(&sched[0], 1u);
            if (wi >= nwork && atomicAdd(&sched[1], 1u) == warps - 1) {
                sched[0] = 0u;
                sched[1] = 0u;
            }
        }
        wi = __shfl_sync(0xffffffffu, wi, 0);
        if (wi >= nwork) break;
        const uint32_t w = list[wi];  // the item's slot: its tile
        const BlockItem it = args.active[w];
        if (args.scenes[it.scene].S != S) {  // never expected: lists are per combination
            if (lane == 0) atomicOr(args.err, ERR_INDEX);
            continue;
        }
        {
            const int4* src = reinterpret_cast<const int4*>(args.scenes + it.scene);
            int4* dst = reinterpret_cast<int4*>(&sc);
            for (int q = lane; q < (int)(sizeof(SceneDev) / 16); q += 32) dst[q] = src[q];
            for (int q = lane; q < W::kTileFloats; q += 32) tile[q] = 0.f;
        }
        __syncwarp();
        const float* pf = sc.buf[args.parity].f;
        const size_t cap = sc.cap;
        const float dt = sc.dt, h = sc.h, inv_h = sc.inv_h;
        const uint32_t i0 = it.start;
        const int count = (int)it.count;
#pragma unroll
        for (int c = 0; c < S; ++c) acc[c].zero();
        int seg_start = 0;     // item index of the open segment's first particle
        int seg_cell = 0;      // its cell
        int cell_start = 0;    // item index of the current cell's first particle
        uint32_t last_cell = 0;  // cell of the previous pass's last particle
        for (int g0 = 0; g0 < count; g0 += W::kStage) {
            const int np = min(W::kStage, count - g0);
            uint32_t cl = 0;
            if (lane < np) {
                p2gStageParticle<S, MODE, W::P, W::WB>(args, sc, pf, cap, dt, h, inv_h, i0 + (uint32_t)(g0 + lane),
                                                       st + lane * W::P);
                cl = args.sorted_keys[i0 + (uint32_t)(g0 + lane)] & 63u;
            }
            // segment starts of this pass: a particle that opens a cell, or
            // one kSeg particles after its cell's first
            uint32_t up = __shfl_up_sync(0xffffffffu, cl, 1);
            if (lane == 0) up = last_cell;
            const unsigned cells = __ballot_sync(0xffffffffu, lane < np && (g0 + lane == 0 || cl != up));
            const unsigned upto = cells & (0xffffffffu >> (31 - lane));  // this lane's and the earlier lanes'
            const int my_cell_start = upto ? g0 + 31 - __clz(upto) : cell_start;
            const unsigned segs = __ballot_sync(0xffffffffu, lane < np && (g0 + lane - my_cell_start) % W::kSeg == 0);
            if (cells) cell_start = g0 + 31 - __clz(cells);
            last_cell = __shfl_sync(0xffffffffu, cl, np - 1);
            const uint32_t cl0 = __shfl_sync(0xffffffffu, cl, 0);
            __syncwarp();  // the staged rows are visible to the warp
            if (g0 == 0) {
                seg_cell = (int)cl0;
            } else if (segs & 1u) {  // the open segment ended with the previous pass
                finish(seg_cell);
                seg_start = g0;
                seg_cell = (int)cl0;
            }
            int qa = 0;
            for (;;) {
                const unsigned rest = segs & ~((2u << qa) - 1u);  // starts after qa
                const int qb = rest ? __ffs(rest) - 1 : np;
                // group grp sums the segment's particles j = grp (mod G), in
                // order, however the segment is cut into passes
                const int jlo = g0 + qa - seg_start;
                if (lane_on) p2gAccumulate<S, MODE, W::P, W::WB, G>(st, qa + (grp - jlo % G + G) % G, qb, na, nb, acc);
                if (qb >= np) break;  // the open segment continues past this pass
                const uint32_t cq = __shfl_sync(0xffffffffu, cl, qb);
                finish(seg_cell);
                seg_start = g0 + qb;
                seg_cell = (int)cq;
                qa = qb;
            }
            __syncwarp();  // the staged rows are read before the next pass overwrites them
        }
        finish(seg_cell);
        float* out = args.tiles + (size_t)w * args.tile_stride;
        for (int q = lane; q < F * TN; q += 32) out[q] = tile[q];
        __syncwarp();  // the tile is read before the next item clears it
    }
    __syncthreads();  // every warp done: the CTA's span ends here
    spanEnd(args.spans, SPAN_P2G, false);
}

// ---------------------------------------------------------------------------
// Grid pass: merge the <= 8 overlapping tiles of every node in fixed order,
// then gravity, v = p/m, v* = v + dt f/m (m > FLT_EPSILON), boundary.
// Node-block N (4^3 nodes starting at 4N-4) is processed by the active block
// B = N - d with the smallest d in {0,1}^3 (x + 2y + 4z order).
// ---------------------------------------------------------------------------
// Barrier of the 64 threads (two warps) of group g of a 256-thread CTA:
// named barrier 1 + g (immediate ids, so the kernel reserves only those).
__device__ __forceinline__ void groupBarrier(int g) {
    switch (g) {
        case 0: asm volatile("bar.sync 1, 64;\n" ::: "memory"); break;
        case 1: asm volatile("bar.sync 2, 64;\n" ::: "memory"); break;
        case 2: asm volatile("bar.sync 3, 64;\n" ::: "memory"); break;
        default: asm volatile("bar.sync 4, 64;\n" ::: "memory"); break;
    }
}

__device__ __forceinline__ int blockSlotAt(const StepArgs& args, const SceneDev& sc, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= sc.nb[0] || y >= sc.nb[1] || z >= sc.nb[2]) return -1;
    return args.block_slot[sc.block_base + (uint32_t)((z * sc.nb[1] + y) * sc.nb[0] + x)];
}

// CTAs per SM: 4 (64 registers) where that costs at most a few bytes of
// spills, else 3 (80 registers): the 8.4M-particle slab's grid pass took
// 0.15 ms at 4 against 0.26 at 3; quadratic APIC and PIC-FLIP spill 36-44
// bytes at 64 registers.
template <int S, int MODE>
struct GridBounds {
    static constexpr int MIN_CTAS = (MODE == MODE_FLIP || (MODE == MODE_APIC_FUSED && S != 4)) ? 3 : 4;
};

template <int S, int MODE>
__global__ void __launch_bounds__(kThreads, GridBounds<S, MODE>::MIN_CTAS) gridKernel(StepArgs args, int want_transfer) {
    constexpr int F = modeFields(MODE);
    constexpr int T = S + 3;
    constexpr int TN = tileNodes(S);
    // A block's merge is a chain of dependent loads.  With at least two work
    // items per CTA, each group of 64 threads merges its own blocks (four in
    // flight per CTA), group g taking items g, g + 4, ... of the CTA's share
    // and synchronising on its own named barrier; with fewer, the whole CTA
    // merges one block, four node blocks at a time.  Per group, the first
    // work item and number of work items of the 3^3 blocks around the
    // current one, index (ox + 1) + 3 (oy + 1) + 9 (oz + 1).
    constexpr int kGroups = kThreads / 64;
    __shared__ int nbSlotAll[kGroups][27], nbItemsAll[kGroups][27];
    const uint32_t nact = args.counters[0];
    const bool grouped = nact >= 2u * gridDim.x;  // uniform over the CTA
    const int ngroups = grouped ? kGroups : 1;
    const int grp = grouped ? (int)(threadIdx.x >> 6) : 0;
    const int gt = grouped ? (int)(threadIdx.x & 63) : (int)threadIdx.x;  // thread within the group
    const int dstep = grouped ? 1 : kGroups;  // node blocks per round
    int* nbSlot = nbSlotAll[grp];
    int* nbItems = nbItemsAll[grp];
    spanBegin(args.spans, SPAN_GRID);
    for (uint32_t w = blockIdx.x * ngroups + grp; w < nact; w += gridDim.x * ngroups) {
        const BlockItem it = args.active[w];
        const SceneDev& sc = args.scenes[it.scene];
        if (sc.S != S || (want_transfer >= 0 && sc.transfer != want_transfer)) continue;
        if (MODE == MODE_MASS && !sc.init_pass) continue;
        if (args.block_slot[it.block] != (int32_t)w) continue;  // a block's first work item does its nodes
        const uint32_t lb = it.block - sc.block_base;
        const int B[3] = {(int)(lb % (uint32_t)sc.nb[0]), (int)((lb / (uint32_t)sc.nb[0]) % (uint32_t)sc.nb[1]),
                          (int)(lb / ((uint32_t)sc.nb[0] * (uint32_t)sc.nb[1]))};
        if (gt < 27) {
            const int o[3] = {gt % 3 - 1, (gt / 3) % 3 - 1, gt / 9 - 1};
            const int slot = blockSlotAt(args, sc, B[0] + o[0], B[1] + o[1], B[2] + o[2]);
            int cnt = 0;
            if (slot >= 0) {
                const uint32_t blk = args.active[slot].block;
                for (uint32_t s2 = (uint32_t)slot; s2 < nact && args.active[s2].block == blk; ++s2) ++cnt;
            }
            nbSlot[gt] = slot;
            nbItems[gt] = cnt;
        }
        if (grouped) groupBarrier(grp);
        else __syncthreads();
#pragma unroll 1
        for (int d0 = 0; d0 < 8; d0 += dstep) {  // the 8 node blocks this block may own
            const int d = d0 + (gt >> 6);
            const int dd[3] = {d & 1, (d >> 1) & 1, (d >> 2) & 1};
            const int N[3] = {B[0] + dd[0], B[1] + dd[1], B[2] + dd[2]};
            if (N[0] >= sc.nb[0] || N[1] >= sc.nb[1] || N[2] >= sc.nb[2]) continue;
            bool owner = true;
            for (int e = 0; e < d && owner; ++e)
                if (nbSlot[(dd[0] - (e & 1) + 1) + 3 * (dd[1] - ((e >> 1) & 1) + 1) + 9 * (dd[2] - ((e >> 2) & 1) + 1)] >= 0)
                    owner = false;
            if (!owner) continue;
            const int l = gt & 63;
            const int L[3] = {l & 3, (l >> 2) & 3, l >> 4};
            const int n[3] = {4 * N[0] - 4 + L[0], 4 * N[1] - 4 + L[1], 4 * N[2] - 4 + L[2]};
            if (n[0] < 0 || n[1] < 0 || n[2] < 0 || n[0] >= sc.res[0] || n[1] >= sc.res[1] || n[2] >= sc.res[2])
                continue;
            float acc[F];
#pragma unroll
            for (int f = 0; f < F; ++f) acc[f] = 0.f;
            // The 8 tiles that overlap the node, in order e, and within each
            // every work item of that block in item order.  The first item's
            // values of Q tiles are loaded together (independent loads in
            // flight), then summed in the same order as one by one.
            constexpr int Q = F <= 4 ? 4 : 2;
#pragma unroll
            for (int hq = 0; hq < 8 / Q; ++hq) {
                float v[Q][F];
                const float* tp[Q];
                int cnt[Q];
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    const int e = Q * hq + q;
                    const int de[3] = {e & 1, (e >> 1) & 1, (e >> 2) & 1};
                    const int ix = L[0] + 4 * de[0], iy = L[1] + 4 * de[1], iz = L[2] + 4 * de[2];
                    const int nbi = (dd[0] - de[0] + 1) + 3 * (dd[1] - de[1] + 1) + 9 * (dd[2] - de[2] + 1);
                    const int slot = (ix < T && iy < T && iz < T) ? nbSlot[nbi] : -1;
                    cnt[q] = slot >= 0 ? nbItems[nbi] : 0;
                    tp[q] = args.tiles + (size_t)(slot >= 0 ? slot : 0) * args.tile_stride + ix + T * (iy + T * iz);
#pragma unroll
                    for (int f = 0; f < F; ++f) v[q][f] = cnt[q] > 0 ? tp[q][f * TN] : 0.f;
                }
                // A block's items are summed first (from its first item's
                // tile), then the block's total is added to the node.
#pragma unroll
                for (int q = 0; q < Q; ++q) {
                    if (cnt[q] <= 0) continue;
                    for (int s2 = 1; s2 < cnt[q]; ++s2) {
                        const float* tile = tp[q] + (size_t)s2 * args.tile_stride;
#pragma unroll
                        for (int f = 0; f < F; ++f) v[q][f] += tile[f * TN];
                    }
#pragma unroll
                    for (int f = 0; f < F; ++f) acc[f] += v[q][f];
                }
            }
            const size_t node = (size_t)n[0] + (size_t)sc.res[0] * ((size_t)n[1] + (size_t)sc.res[1] * n[2]);
            const size_t nodes = (size_t)sc.res[0] * sc.res[1] * sc.res[2];
            if (MODE == MODE_SPLIT) {
                float* dbg = sc.dbg;
                dbg[node] += acc[0];
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    dbg[(1 + a) * nodes + node] += acc[1 + a];
                    dbg[(4 + a) * nodes + node] += acc[4 + a];
                }
                continue;
            }
            if (MODE == MODE_MASS) {
                sc.vstar[node] = make_float4(0.f, 0.f, 0.f, acc[0]);
                continue;
            }
            const float m = acc[0], dt = sc.dt;
            if (m > 0.f) atomicAdd(&args.stats[2], 1u);
            float vs[3] = {0.f, 0.f, 0.f}, vo[3] = {0.f, 0.f, 0.f};
            if (MODE == MODE_APIC_FUSED) {
                if (m > kFltEps) {
#pragma unroll
                    for (int a = 0; a < 3; ++a) vs[a] = __fdiv_rn(acc[1 + a], m);
                    vs[1] -= dt * sc.gravity;
                }
            } else {  // MODE_FLIP
                if (m > kFltEps) {
                    float fy = acc[5] - sc.gravity * m;
                    const float fo[3] = {acc[4], fy, acc[6]};
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        vo[a] = __fdiv_rn(acc[1 + a], m);
                        vs[a] = vo[a] + __fdiv_rn(dt * fo[a], m);
                    }
                } else {
#pragma unroll
                    for (int a = 0; a < 3; ++a) vo[a] = acc[1 + a];
                }
            }
            if (sc.boundary == MPM_BOUNDARY_STICKY) {
                bool wall = false;
#pragma unroll
                for (int a = 0; a < 3; ++a) wall |= (n[a] < sc.sticky) || (n[a] >= sc.res[a] - sc.sticky);
                if (wall) vs[0] = vs[1] = vs[2] = 0.f;
            } else {
                float pos[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) pos[a] = (sc.origin[a] + sc.h * (float)n[a]) + dt * vs[a];
                boundaryCollision(pos, vs, sc.origin, sc.target, sc.friction);
            }
            if (sc.phi) {
                float pos[3];
#pragma unroll
                for (int a = 0; a < 3; ++a) pos[a] = (sc.origin[a] + sc.h * (float)n[a]) + dt * vs[a];
                levelSetCollision(sc, pos, vs);
            }
            sc.vstar[node] = make_float4(vs[0], vs[1], vs[2], m);
            if (MODE == MODE_FLIP) sc.vold[node] = make_float4(vo[0], vo[1], vo[2], 0.f);
        }
        if (grouped) groupBarrier(grp);  // the neighbour table is rewritten for the next item
        else __syncthreads();
    }
    __syncthreads();  // every group done: the CTA's span ends here
    spanEnd(args.spans, SPAN_GRID);
}

// ---------------------------------------------------------------------------
// G2P, fused with the particle update.  One CTA per active block: the block's
// (S+3)^3 node tile of v* (and v) is staged in shared memory, then one thread
// per particle.  Writes the particle to its sorted slot of the other buffer.
// ---------------------------------------------------------------------------
// The first loads of a particle's update, issued one particle ahead: the
// permutation entry, x and v into registers, and Fe, Fp, V0 into the thread's
// shared-memory row by cp.async (one commit group per particle, possibly
// empty), so their latency overlaps the previous particle's update.
struct G2PIn {
    uint32_t old;
    bool ok;
    float x[3], v[3];
};
__device__ __forceinline__ G2PIn g2pFetch(const StepArgs& args, const SceneDev& sc, uint32_t gs, float* pre) {
    G2PIn p;
    const float* pf = sc.buf[args.parity].f;
    const size_t cap = sc.cap;
    const uint32_t old = args.perm[gs] - sc.key_offset;
    const uint32_t dst = gs - sc.key_offset;
    p.ok = old < sc.n && dst < sc.n;  // range check: never expected, skip instead of faulting
    p.old = p.ok ? old : 0u;
    if (p.ok) {
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            cpAsync4(pre + k, pf + (F_FE + k) * cap + old);
            cpAsync4(pre + 9 + k, pf + (F_FP + k) * cap + old);
        }
        cpAsync4(pre + 18, pf + F_VOL * cap + old);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            p.x[a] = ldg(pf + (F_X + a) * cap + old);
            p.v[a] = ldg(pf + (F_V + a) * cap + old);
        }
    } else {
        atomicOr(args.err, ERR_INDEX);
    }
    cpAsyncCommit();
    return p;
}
__device__ __forceinline__ void cpAsyncWaitPrevious() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int S, bool APIC>
__device__ __forceinline__ void particleUpdate(const StepArgs& args, const SceneDev& sc, uint32_t gs, const G2PIn& in,
                                               bool next_pending, const float4* tvs, const float4* tvo, const int* t0,
                                               bool fused, float* pre, const MaterialDev& mat0) {
    constexpr int T = S + 3;
    const float* pf = sc.buf[args.parity].f;
    float* nf = sc.buf[args.parity ^ 1].f;
    const size_t cap = sc.cap;
    if (!in.ok) {
        if (next_pending) cpAsyncWaitPrevious();
        else cpAsyncWaitAll();
        return;
    }
    const uint32_t old = in.old;
    const uint32_t dst = gs - sc.key_offset;
    const float h = sc.h, dt = sc.dt;
    float x[3], v[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        x[a] = in.x[a];
        v[a] = in.v[a];
    }
    float vpic[3] = {0.f, 0.f, 0.f}, dflip[3] = {0.f, 0.f, 0.f};
    float gv[9], K[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) gv[k] = K[k] = 0.f;
    float delta[3] = {0.f, 0.f, 0.f};
    int base[3];
    bool in_tile = false;
    if (tvs) {
        in_tile = stencilBase(sc, x, base);
#pragma unroll
        for (int a = 0; a < 3; ++a) in_tile = in_tile && base[a] - t0[a] >= 0 && base[a] - t0[a] <= 3;
        if (!in_tile) atomicOr(args.err, ERR_INDEX);  // key and position disagree: never expected
    }
    if (in_tile) {
        float w[3][S], dw[3][S];
        int lo[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = base[a] - t0[a];
            float gp0 = __fadd_rn(sc.origin[a], __fmul_rn(h, (float)base[a]));
            delta[a] = x[a] - gp0;
            float dk[S];
            dk[0] = __fdiv_rn(delta[a], h);
#pragma unroll
            for (int k = 1; k < S; ++k) dk[k] = dk[0] - (float)k;  // exact subtraction
            splineWeights<S>(dk, w[a], dw[a]);
#pragma unroll
            for (int k = 0; k < S; ++k) {
                dw[a][k] *= sc.inv_h;
            }
        }
        // Separable gather in packed FP32 pairs: the x and y components of
        // every sum go through one __ffma2_rn (two exactly rounded FMAs, the
        // same results as fmaf), z through fmaf.  Column j of grad v and of
        // the APIC moment K is held as (row 0, row 1) pair + row 2.
        float2 wp[S], dwp[S], wap[S];
#pragma unroll
        for (int a = 0; a < S; ++a) {
            wp[a] = make_float2(w[0][a], w[0][a]);
            dwp[a] = make_float2(dw[0][a], dw[0][a]);
            const float wa = w[0][a] * (float)a;
            wap[a] = make_float2(wa, wa);
        }
        float2 vp_xy = make_float2(0.f, 0.f), df_xy = make_float2(0.f, 0.f), gv_xy[3], K_xy[3];
        float vp_z = 0.f, df_z = 0.f, gv_z[3], K_z[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            gv_xy[j] = K_xy[j] = make_float2(0.f, 0.f);
            gv_z[j] = K_z[j] = 0.f;
        }
#pragma unroll
        for (int c = 0; c < S; ++c) {
#pragma unroll
            for (int b = 0; b < S; ++b) {
                float2 r0 = make_float2(0.f, 0.f), r1 = r0, rd = r0, rv = r0;
                float r0z = 0.f, r1z = 0.f, rdz = 0.f, rvz = 0.f;
                const int rowbase = lo[0] + T * ((lo[1] + b) + T * (lo[2] + c));
#pragma unroll
                for (int a = 0; a < S; ++a) {
                    const float4 g = tvs[rowbase + a];
                    const float2 gxy = make_float2(g.x, g.y);
                    r0 = __ffma2_rn(wp[a], gxy, r0);
                    r0z = fmaf(w[0][a], g.z, r0z);
                    rd = __ffma2_rn(dwp[a], gxy, rd);
                    rdz = fmaf(dw[0][a], g.z, rdz);
                    if (APIC) {
                        r1 = __ffma2_rn(wap[a], gxy, r1);
                        r1z = fmaf(wap[a].x, g.z, r1z);
                    } else {
                        const float4 o = tvo[rowbase + a];
                        const float2 d = __fadd2_rn(gxy, make_float2(-o.x, -o.y));  // g - o, exactly
                        rv = __ffma2_rn(wp[a], d, rv);
                        rvz = fmaf(w[0][a], g.z - o.z, rvz);
                    }
                }
                const float wyz = w[1][b] * w[2][c];
                const float dy = dw[1][b] * w[2][c];
                const float dz = w[1][b] * dw[2][c];
                const float2 wyz2 = make_float2(wyz, wyz), dy2 = make_float2(dy, dy), dz2 = make_float2(dz, dz);
                vp_xy = __ffma2_rn(wyz2, r0, vp_xy);
                vp_z = fmaf(wyz, r0z, vp_z);
                gv_xy[0] = __ffma2_rn(wyz2, rd, gv_xy[0]);
                gv_z[0] = fmaf(wyz, rdz, gv_z[0]);
                gv_xy[1] = __ffma2_rn(dy2, r0, gv_xy[1]);
                gv_z[1] = fmaf(dy, r0z, gv_z[1]);
                gv_xy[2] = __ffma2_rn(dz2, r0, gv_xy[2]);
                gv_z[2] = fmaf(dz, r0z, gv_z[2]);
                if (APIC) {
                    const float wb = wyz * (float)b, wc = wyz * (float)c;
                    K_xy[0] = __ffma2_rn(wyz2, r1, K_xy[0]);
                    K_z[0] = fmaf(wyz, r1z, K_z[0]);
                    K_xy[1] = __ffma2_rn(make_float2(wb, wb), r0, K_xy[1]);
                    K_z[1] = fmaf(wb, r0z, K_z[1]);
                    K_xy[2] = __ffma2_rn(make_float2(wc, wc), r0, K_xy[2]);
                    K_z[2] = fmaf(wc, r0z, K_z[2]);
                } else {
                    df_xy = __ffma2_rn(wyz2, rv, df_xy);
                    df_z = fmaf(wyz, rvz, df_z);
                }
            }
        }
        vpic[0] = vp_xy.x;
        vpic[1] = vp_xy.y;
        vpic[2] = vp_z;
        dflip[0] = df_xy.x;
        dflip[1] = df_xy.y;
        dflip[2] = df_z;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            gv[0 * 3 + j] = gv_xy[j].x;
            gv[1 * 3 + j] = gv_xy[j].y;
            gv[2 * 3 + j] = gv_z[j];
            K[0 * 3 + j] = K_xy[j].x;
            K[1 * 3 + j] = K_xy[j].y;
            K[2 * 3 + j] = K_z[j];
        }
    }
    // New velocity (src/mpm_solver3d.cu:362-363; apic :366-374).
    float vn[3];
    if (APIC) {
#pragma unroll
        for (int i = 0; i < 3; ++i) vn[i] = vpic[i];
    } else {
        const float al = sc.blend, om = 1.0f - sc.blend;
#pragma unroll
        for (int i = 0; i < 3; ++i) vn[i] = al * (v[i] + dflip[i]) + om * vpic[i];
    }
    // Fe <- (I + dt grad v) Fe ; F = Fe Fp ; SVD clamp (src/material_point3d.cu:53-70).
    float Fe[9], Fp[9], A[9], Fn[9];
    if (next_pending) cpAsyncWaitPrevious();  // this particle's group; the next one's may still run
    else cpAsyncWaitAll();
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        Fe[k] = pre[k];
        Fp[k] = pre[9 + k];
        A[k] = dt * gv[k] + ((k % 4 == 0) ? 1.0f : 0.0f);
    }
    matmul3(A, Fe, Fn);
    const uint16_t mid = sc.nmat > 1 ? sc.buf[args.parity].mat[old] : (uint16_t)0;
    const MaterialDev m = sc.nmat > 1 ? sc.mats[mid] : mat0;
    const float hi = 1.0f + m.theta_s, lo = 1.0f - m.theta_c;
    const float V0 = pre[18];
    float mu, la, tau[6];
    // Elastic fast path: no singular value can be clamped, so Fe = Fn and Fp
    // stay as they are, and the stress comes from the polar rotation of Fn
    // (no SVD).  Material bounds beyond 25 % always take the SVD path.
    const float theta = fmaxf(m.theta_s, m.theta_c);
    if (theta <= 0.25f && singularValuesInside(Fn, lo, hi)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) Fe[k] = Fn[k];
        plasticLame(m, Fp, mu, la);
        const float J = det3(Fn);
        float P[9];  // 2 mu (F - R) for fixed corotated, mu F for Neo-Hookean
        float diag;
        if (m.model == MPM_MODEL_NEO_HOOKEAN) {
#pragma unroll
            for (int k = 0; k < 9; ++k) P[k] = mu * Fn[k];
            diag = la * logf(J) - mu;
        } else {
            float R[9];
            polarRotation(Fn, R, theta <= 0.1f ? 3 : 4);
#pragma unroll
            for (int k = 0; k < 9; ++k) P[k] = 2.0f * mu * (Fn[k] - R[k]);
            diag = la * (J - 1.0f) * J;
        }
        const int I[6] = {0, 1, 2, 0, 0, 1}, Jx[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
        for (int e = 0; e < 6; ++e) {
            const int i = I[e], j = Jx[e];
            float v = fmaf(P[3 * i + 2], Fn[3 * j + 2], fmaf(P[3 * i + 1], Fn[3 * j + 1], P[3 * i] * Fn[3 * j]));
            if (e < 3) v += diag;
            tau[e] = V0 * v;
        }
    } else {
    float U[9], V[9], s[3];
    svd3(Fn, U, s, V);
    bool clamped = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float c = fmaxf(fminf(s[k], hi), lo);
        clamped |= c != s[k];
        s[k] = c;
    }
    if (clamped) {
        // Fe = U S V^T ; Fp = V S^-1 U^T (Fe Fp)
        float Ff[9];
        matmul3(Fn, Fp, Ff);
        float US[9], VSi[9];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                US[3 * i + k] = U[3 * i + k] * s[k];
                VSi[3 * i + k] = V[3 * i + k] / s[k];
            }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                Fe[3 * i + j] = US[3 * i] * V[3 * j] + US[3 * i + 1] * V[3 * j + 1] + US[3 * i + 2] * V[3 * j + 2];
                A[3 * i + j] = VSi[3 * i] * U[3 * j] + VSi[3 * i + 1] * U[3 * j + 1] + VSi[3 * i + 2] * U[3 * j + 2];
            }
        matmul3(A, Ff, Fp);
    } else {
        // No singular value clamped: U S V^T = Fn and V S^-1 U^T Fn Fp = Fp in
        // exact arithmetic; keeping Fn and Fp avoids the FP32 SVD round-off.
#pragma unroll
        for (int k = 0; k < 9; ++k) Fe[k] = Fn[k];
    }
    // Next step's stress from the clamped SVD (Fe = U S V^T exactly).
    plasticLame(m, Fp, mu, la);
    if (m.model == MPM_MODEL_NEO_HOOKEAN) {
        bool proj = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            proj |= s[k] < kFltEps;
            s[k] = fmaxf(s[k], kFltEps);
        }
        if (proj)
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j)
                    Fe[3 * i + j] = U[3 * i] * s[0] * V[3 * j] + U[3 * i + 1] * s[1] * V[3 * j + 1] +
                                    U[3 * i + 2] * s[2] * V[3 * j + 2];
    }
    tauFromSvd(m.model, U, s, mu, la, V0, tau);
    }
    if (fused) {
        if (sc.pcoll) {  // particlesCollision (src/mpm_solver3d.cu:428-445)
            float pos[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) pos[a] = x[a] + dt * vn[a];
            boundaryCollision(pos, vn, sc.origin, sc.target, sc.friction);
            if (sc.phi) {
#pragma unroll
                for (int a = 0; a < 3; ++a) pos[a] = x[a] + dt * vn[a];
                levelSetCollision(sc, pos, vn);
            }
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) x[a] += dt * vn[a];  // advectParticles (:381-391)
        const uint32_t key = particleKey(sc, x, args.err);
        args.next_keys[gs] = key;
        // one atomic per distinct block among the converged lanes (sorted
        // particles: a warp's lanes nearly always share their next block)
        const uint32_t blk = key >> 6;
        const uint32_t peers = __match_any_sync(__activemask(), blk);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&args.block_count[blk], (uint32_t)__popc(peers));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        nf[(F_X + a) * cap + dst] = x[a];
        nf[(F_V + a) * cap + dst] = vn[a];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        nf[(F_FE + k) * cap + dst] = Fe[k];
        nf[(F_FP + k) * cap + dst] = Fp[k];
    }
    if (APIC) {
        // B = sum w v* (x_i - x_p)^T = h K - vpic delta^T
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) nf[(F_B + 3 * i + j) * cap + dst] = h * K[3 * i + j] - vpic[i] * delta[j];
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) nf[(F_TAU + k) * cap + dst] = tau[k];
    nf[F_MASS * cap + dst] = ldg(pf + F_MASS * cap + old);
    nf[F_VOL * cap + dst] = V0;
    sc.buf[args.parity ^ 1].pid[dst] = sc.buf[args.parity].pid[old];
    if (sc.nmat > 1) sc.buf[args.parity ^ 1].mat[dst] = mid;
}

// ---------------------------------------------------------------------------
// TMA (cp.async.bulk.tensor) and mbarrier helpers for G2P's grid tile.  The
// tensor map of a scene's dense float4 grid is 4-D FP32: (component, x, y, z),
// so the innermost box extent is one node's 16 bytes and every tile origin is
// aligned whatever its x; nodes outside the grid read as zeros (OOB fill).
// The maps cover this GPU's own grid memory; there is no multicast.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbarInitFence() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smemAddr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Orders this CTA's earlier generic-proxy accesses of shared memory before
// later async-proxy (TMA) writes to it.
__device__ __forceinline__ void fenceProxyAsyncShared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tensorMapAcquire(const void* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
}
// Box of the 4-D map at (0, x, y, z) into dst, completing on bar.
__device__ __forceinline__ void tmaLoadTile(void* dst, const void* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smemAddr(dst)),
        "l"(map), "r"(0), "r"(x), "r"(y), "r"(z), "r"(smemAddr(bar))
        : "memory");
}

// Bounded wait on an mbarrier phase: gives up after ~2^22 polls (seconds),
// raising ERR_WAIT_TIMEOUT and setting *abort (when given) so that the CTA's
// other waiters give up too (they look at it every 256 polls).  Returns false
// when it gave up.
__device__ __forceinline__ bool waitTile(uint64_t* bar, unsigned parity, uint32_t* err, volatile int* abort) {
    for (uint32_t i = 0; !mbarTryWait(bar, parity); ++i) {
        if (i > (1u << 22)) {
            atomicOr(err, ERR_WAIT_TIMEOUT);
            if (abort) *abort = 1;
            return false;
        }
        if (abort && (i & 255u) == 255u && *abort) return false;
        if (i > 64) __nanosleep(64);
    }
    return true;
}

// Origin (node index) of the (S+3)^3 tile of an active block: 4 B - 4 per axis.
__device__ __forceinline__ void tileOrigin(const SceneDev& sc, uint32_t block, int* t0) {
    const uint32_t lb = block - sc.block_base;
    t0[0] = 4 * (int)(lb % (uint32_t)sc.nb[0]) - 4;
    t0[1] = 4 * (int)((lb / (uint32_t)sc.nb[0]) % (uint32_t)sc.nb[1]) - 4;
    t0[2] = 4 * (int)(lb / ((uint32_t)sc.nb[0] * (uint32_t)sc.nb[1])) - 4;
}

// Bulk copy (cp.async.bulk) of bytes from global to shared memory, completing
// on bar; both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulkLoad(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smemAddr(bar)) : "memory");
}

// G2P: persistent CTAs take work items from this combination's list (then the
// outside items).  One elected thread produces: it fetches the next item and
// copies, by TMA, the item's tile of v* (and v), its scene entry and the
// scene's first material into one of two shared-memory slots, completing on
// the slot's "full" mbarrier.  Every warp consumes: it waits on "full",
// updates its particles of the item and arrives on the slot's "empty"
// mbarrier; the producer refills a slot only when all warps have released it.
// So warps run up to one item apart instead of meeting at a CTA barrier after
// every item, and the particle update reads the scene and material from
// shared memory.
// Resident G2P CTAs per SM the register budget is fitted to: 2 gives 128
// registers a thread and no spills (two-ball G2P 0.132 -> 0.117 ms against 3
// CTAs at 80 registers, which spill ~150 bytes a thread).
#ifndef MPM_G2P_THREADS
#define MPM_G2P_THREADS 256
#endif
constexpr int kG2PThreads = MPM_G2P_THREADS;
constexpr int kG2PWarps = kG2PThreads / 32;
#ifndef MPM_G2P_MIN_CTAS
#define MPM_G2P_MIN_CTAS (2 * 256 / MPM_G2P_THREADS)
#endif
template <int S, bool APIC>
__global__ void __launch_bounds__(kG2PThreads, MPM_G2P_MIN_CTAS) g2pKernel(StepArgs args, int fused) {
    constexpr int T = S + 3;
    constexpr int TN = tileNodes(S);
    constexpr int TNP = (TN + 7) & ~7;  // buffers 128-byte aligned
    constexpr unsigned kTileBytes = (unsigned)TN * 16u;
    static_assert(sizeof(SceneDev) % 16 == 0 && sizeof(MaterialDev) % 16 == 0, "bulk copies need 16-byte sizes");
    __shared__ __align__(128) float4 tvs[2][TNP];
    __shared__ __align__(128) float4 tvo[APIC ? 1 : 2][APIC ? 8 : TNP];
    // two per-thread prefetch rows of Fe, Fp, V0 (dynamic shared memory: with
    // the tiles they exceed the 48 KB of static shared memory)
    extern __shared__ float4 g2p_dyn[];
    float (*pre)[kG2PThreads * kPreStride] = reinterpret_cast<float (*)[kG2PThreads * kPreStride]>(g2p_dyn);
    __shared__ SceneDev scs[2];
    __shared__ MaterialDev mat0[2];
    __shared__ BlockItem its[2];
    __shared__ uint32_t item_s[2];
    __shared__ __align__(8) uint64_t full[2], empty[2];
    const int want = APIC ? MPM_TRANSFER_APIC : MPM_TRANSFER_PIC_FLIP;
    // this combination's own (finer) items of the active blocks, then the
    // outside items of all scenes (the others' are skipped)
    const uint32_t nact = args.counters[kG2PCountWord + args.combo];
    const BlockItem* items = args.g2p_items + (size_t)args.combo * args.g2p_cap;
    const uint32_t nout = args.counters[1];
    const uint32_t total = nact + nout;
    uint32_t* sched = args.sched + 4;
    const int lane = threadIdx.x & 31;

    // Producer (thread 0): the next item (the last CTA to run out clears the
    // scheduler, so every launch starts from zero) into slot b -- its scene
    // entry, the scene's first material and, for an active block, the tile
    // of v* (and v) -- completing on full[b].  After the first index past the
    // end it only hands out the end marker.
    bool ran_out = false;
    auto produce = [&](int b) {
        uint32_t w = total;
        if (!ran_out) {
            w = atomicAdd(&sched[0], 1u);
            if (w >= total) {
                ran_out = true;
                if (atomicAdd(&sched[1], 1u) == gridDim.x - 1) {
                    sched[0] = 0u;
                    sched[1] = 0u;
                }
            }
        }
        item_s[b] = w;
        if (w >= total) {
            mbarArrive(&full[b]);
            return;
        }
        const BlockItem it = w < nact ? items[w] : args.outside[w - nact];
        its[b] = it;
        const SceneDev* sg = args.scenes + it.scene;
        const bool tile = w < nact;
        fenceProxyAsyncShared();  // the slot's earlier generic reads come first
        mbarExpectTx(&full[b], (unsigned)(sizeof(SceneDev) + sizeof(MaterialDev)) +
                                   (tile ? (APIC ? kTileBytes : 2u * kTileBytes) : 0u));
        bulkLoad(&scs[b], sg, (unsigned)sizeof(SceneDev), &full[b]);
        bulkLoad(&mat0[b], sg->mats, (unsigned)sizeof(MaterialDev), &full[b]);
        if (tile) {
            int t0[3];
            tileOrigin(*sg, it.block, t0);
            const unsigned char* maps = args.tmaps + (size_t)it.scene * 2 * kTensorMapBytes;
            tensorMapAcquire(maps);
            tmaLoadTile(&tvs[b][0], maps, t0[0], t0[1], t0[2], &full[b]);
            if (!APIC) {
                tensorMapAcquire(maps + kTensorMapBytes);
                tmaLoadTile(&tvo[b][0], maps + kTensorMapBytes, t0[0], t0[1], t0[2], &full[b]);
            }
        }
    };
    // A wait that gives up (never expected) sets abort_s: the producer stops
    // issuing copies, every warp leaves the loop at its next slot wait (as a
    // whole warp), and thread 0 waits for the copies still in flight before
    // the CTA exits, so that none lands in shared memory it no longer owns.
    __shared__ int abort_s;
    spanBegin(args.spans, SPAN_G2P);
    if (threadIdx.x == 0) {
        abort_s = 0;
        mbarInit(&full[0], 1);
        mbarInit(&full[1], 1);
        mbarInit(&empty[0], kG2PWarps);
        mbarInit(&empty[1], kG2PWarps);
        mbarInitFence();
        produce(0);
    }
    __syncthreads();
    unsigned full_ph = 0u, empty_ph = 0u;  // bit b: parity of slot b's next wait
    unsigned issued = 1u;                  // thread 0: slots whose copies it has not yet seen land
    for (int k = 0, b = 0;; ++k, b ^= 1) {
        if (threadIdx.x == 0 && !abort_s) {
            // slot b ^ 1 gets item k + 1; it held item k - 1
            bool free_slot = true;
            if (k >= 1) {
                free_slot = waitTile(&empty[b ^ 1], (empty_ph >> (b ^ 1)) & 1u, args.err, &abort_s);
                if (free_slot) empty_ph ^= 1u << (b ^ 1);
            }
            if (free_slot) {
                produce(b ^ 1);
                issued |= 1u << (b ^ 1);
            }
        }
        const bool landed = waitTile(&full[b], (full_ph >> b) & 1u, args.err, &abort_s);
        if (__any_sync(0xffffffffu, !landed)) break;  // gave up (never expected): the whole warp leaves
        if (threadIdx.x == 0) issued &= ~(1u << b);
        full_ph ^= 1u << b;
        const uint32_t w = item_s[b];
        if (w >= total) break;
        const bool inside = w < nact;
        const BlockItem it = its[b];
        const SceneDev& sc = scs[b];
        int t0[3] = {0, 0, 0};
        if (inside) tileOrigin(sc, it.block, t0);
        if ((inside || (sc.S == S && sc.transfer == want)) && threadIdx.x < it.count) {
            // each thread's particles of the item, the next one's loads in
            // flight during the current one's update (rows alternate)
            int row = 0;
            G2PIn cur = g2pFetch(args, sc, it.start + threadIdx.x, &pre[0][threadIdx.x * kPreStride]);
            for (uint32_t i = threadIdx.x; i < it.count; i += kG2PThreads) {
                const bool more = i + kG2PThreads < it.count;
                G2PIn nxt;
                if (more) nxt = g2pFetch(args, sc, it.start + i + kG2PThreads, &pre[row ^ 1][threadIdx.x * kPreStride]);
                particleUpdate<S, APIC>(args, sc, it.start + i, cur, more, inside ? &tvs[b][0] : nullptr,
                                        APIC ? nullptr : &tvo[b][0], t0, fused != 0,
                                        &pre[row][threadIdx.x * kPreStride], mat0[b]);
                if (more) cur = nxt;
                row ^= 1;
            }
        }
        __syncwarp();
        if (lane == 0) mbarArrive(&empty[b]);
    }
    if (threadIdx.x == 0 && abort_s) {
        // copies issued and not seen landing: wait for them, bounded again
        for (int s = 0; s < 2; ++s)
            if ((issued >> s) & 1u) waitTile(&full[s], (full_ph >> s) & 1u, args.err, nullptr);
    }
    __syncthreads();  // every warp done: the CTA's span ends here
    spanEnd(args.spans, SPAN_G2P);
}

// ---------------------------------------------------------------------------
// Split-mode dense grid kernels on sc.dbg planes: mass, vel[3], force[3], vstar[3].
// ---------------------------------------------------------------------------
__global__ void denseGravityKernel(const SceneDev* __restrict__ scenes) {
    const SceneDev& sc = scenes[blockIdx.y];
    const size_t nodes = (size_t)sc.res[0] * sc.res[1] * sc.res[2];
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < nodes; i += (size_t)gridDim.x * kThreads) {
        float m = sc.dbg[i];
        if (m > kFltEps) sc.dbg[5 * nodes + i] -= sc.gravity * m;  // force.y
    }
}

__global__ void denseUpdateVelocityKernel(const SceneDev* __restrict__ scenes, float dt) {
    const SceneDev& sc = scenes[blockIdx.y];
    const size_t nodes = (size_t)sc.res[0] * sc.res[1] * sc.res[2];
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < nodes; i += (size_t)gridDim.x * kThreads) {
        float m = sc.dbg[i];
        if (m > kFltEps) {
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                float v = __fdiv_rn(sc.dbg[(1 + a) * nodes + i], m);
                sc.dbg[(1 + a) * nodes + i] = v;
                sc.dbg[(7 + a) * nodes + i] = v + __fdiv_rn(dt * sc.dbg[(4 + a) * nodes + i], m);
            }
        }
    }
}

__global__ void denseCollisionKernel(const SceneDev* __restrict__ scenes, float dt) {
    const SceneDev& sc = scenes[blockIdx.y];
    const size_t nodes = (size_t)sc.res[0] * sc.res[1] * sc.res[2];
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < nodes; i += (size_t)gridDim.x * kThreads) {
        const int n[3] = {(int)(i % sc.res[0]), (int)((i / sc.res[0]) % sc.res[1]),
                          (int)(i / ((size_t)sc.res[0] * sc.res[1]))};
        float vs[3] = {sc.dbg[7 * nodes + i], sc.dbg[8 * nodes + i], sc.dbg[9 * nodes + i]};
        if (sc.boundary == MPM_BOUNDARY_STICKY) {
            bool wall = false;
#pragma unroll
            for (int a = 0; a < 3; ++a) wall |= (n[a] < sc.sticky) || (n[a] >= sc.res[a] - sc.sticky);
            if (wall) vs[0] = vs[1] = vs[2] = 0.f;
        } else {
            float pos[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) pos[a] = (sc.origin[a] + sc.h * (float)n[a]) + dt * vs[a];
            boundaryCollision(pos, vs, sc.origin, sc.target, sc.friction);
        }
        if (sc.phi) {
            float pos[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) pos[a] = (sc.origin[a] + sc.h * (float)n[a]) + dt * vs[a];
            levelSetCollision(sc, pos, vs);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) sc.dbg[(7 + a) * nodes + i] = vs[a];
    }
}

// dbg planes -> float4 v*, v for the G2P kernel.
__global__ void densePackKernel(const SceneDev* __restrict__ scenes) {
    const SceneDev& sc = scenes[blockIdx.y];
    const size_t nodes = (size_t)sc.res[0] * sc.res[1] * sc.res[2];
    for (size_t i = (size_t)blockIdx.x * kThreads + threadIdx.x; i < nodes; i += (size_t)gridDim.x * kThreads) {
        sc.vstar[i] = make_float4(sc.dbg[7 * nodes + i], sc.dbg[8 * nodes + i], sc.dbg[9 * nodes + i], sc.dbg[i]);
        if (sc.vold)
            sc.vold[i] = make_float4(sc.dbg[nodes + i], sc.dbg[2 * nodes + i], sc.dbg[3 * nodes + i], 0.f);
    }
}

__global__ void particlesCollisionKernel(const SceneDev* __restrict__ scenes, int parity, float dt) {
    const SceneDev& sc = scenes[blockIdx.y];
    float* f = sc.buf[parity].f;
    const size_t cap = sc.cap;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads) {
        float x[3], v[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            v[a] = f[(F_V + a) * cap + i];
            x[a] = f[(F_X + a) * cap + i] + dt * v[a];
        }
        boundaryCollision(x, v, sc.origin, sc.target, sc.friction);
        if (sc.phi) {
#pragma unroll
            for (int a = 0; a < 3; ++a) x[a] = f[(F_X + a) * cap + i] + dt * v[a];
            levelSetCollision(sc, x, v);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) f[(F_V + a) * cap + i] = v[a];
    }
}

__global__ void advectKernel(const SceneDev* __restrict__ scenes, int parity, float dt) {
    const SceneDev& sc = scenes[blockIdx.y];
    float* f = sc.buf[parity].f;
    const size_t cap = sc.cap;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads)
#pragma unroll
        for (int a = 0; a < 3; ++a) f[(F_X + a) * cap + i] += dt * f[(F_V + a) * cap + i];
}

// Particle state of a new scene from the caller's arrays staged on the device
// as [x: 3n interleaved][v: 3n interleaved][m: n][V0: n, prescribed only]:
// SoA planes with Fe = Fp = I, B = tau = 0 and V0 = 0 unless prescribed
// (the reference's MaterialPoint3D constructor, src/material_point3d.cu:10-30).
// With `perm` slot i takes the caller's particle perm[i] (the cell-sorted
// order), else particle i; pid records it.  mat_in: the caller's material ids
// (staged), else none.
__global__ void initStateKernel(float* __restrict__ f, uint32_t* __restrict__ pid, uint16_t* __restrict__ mat,
                                size_t cap, const float* __restrict__ staged, size_t n, int has_volume,
                                const uint32_t* __restrict__ perm, const uint16_t* __restrict__ mat_in) {
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kThreads) {
        const size_t o = perm ? (size_t)perm[i] : i;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            f[(F_X + a) * cap + i] = staged[3 * o + a];
            f[(F_V + a) * cap + i] = staged[3 * n + 3 * o + a];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            f[(F_FE + k) * cap + i] = (k % 4 == 0) ? 1.f : 0.f;
            f[(F_FP + k) * cap + i] = (k % 4 == 0) ? 1.f : 0.f;
            f[(F_B + k) * cap + i] = 0.f;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) f[(F_TAU + k) * cap + i] = 0.f;
        f[F_MASS * cap + i] = staged[6 * n + o];
        f[F_VOL * cap + i] = has_volume ? staged[7 * n + o] : 0.f;
        pid[i] = (uint32_t)o;
        if (mat_in) mat[i] = mat_in[o];
    }
}

// Cell keys of a new scene's staged positions (caller order, x y z
// interleaved), for the cell-sorted initial order.
__global__ void __launch_bounds__(kThreads) stagedKeyKernel(const SceneDev sc, const float* __restrict__ xyz,
                                                             uint32_t n, uint32_t* __restrict__ keys,
                                                             uint32_t* __restrict__ err) {
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const float x[3] = {xyz[3 * (size_t)i], xyz[3 * (size_t)i + 1], xyz[3 * (size_t)i + 2]};
        keys[i] = particleKey(sc, x, err);
    }
}

// initialize(): V0 = m / (sum_i m_i w_ip / h^3) with node masses in vstar.w
// (src/mpm_solver3d.cu:173-214).  Live order, dense node reads.
template <int S>
__global__ void volumeKernel(const SceneDev* __restrict__ scenes, int parity) {
    const SceneDev& sc = scenes[blockIdx.y];
    float* f = sc.buf[parity].f;
    const size_t cap = sc.cap;
    const float h = sc.h;
    const float inv_cell_vol = (float)(1.0 / (double)(h * h * h));
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads) {
        float x[3] = {f[F_X * cap + i], f[(F_X + 1) * cap + i], f[(F_X + 2) * cap + i]};
        int base[3];
        float dens = 0.f;
        if (stencilBase(sc, x, base)) {
            float w[3][S];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int k = 0; k < S; ++k) {
                    float gp = __fadd_rn(sc.origin[a], __fmul_rn(h, (float)(base[a] + k)));
                    w[a][k] = splineN<S>(__fdiv_rn(__fsub_rn(x[a], gp), h));
                }
            // nodes in the grid per axis (all of them but at the edges); the
            // sum runs over the stencil in the same order either way
            bool in[3][S];
#pragma unroll
            for (int a = 0; a < 3; ++a)
#pragma unroll
                for (int k = 0; k < S; ++k) in[a][k] = base[a] + k >= 0 && base[a] + k < sc.res[a];
            const size_t X = (size_t)sc.res[0], XY = X * (size_t)sc.res[1];
            const float* mass = reinterpret_cast<const float*>(sc.vstar) + 3;  // vstar[node].w
            const long long n0 = (long long)base[0] + (long long)X * base[1] + (long long)XY * base[2];
#pragma unroll
            for (int c = 0; c < S; ++c)
#pragma unroll
                for (int b = 0; b < S; ++b)
#pragma unroll
                    for (int a = 0; a < S; ++a) {
                        if (!(in[0][a] && in[1][b] && in[2][c])) continue;
                        const size_t node = (size_t)(n0 + a + (long long)X * b + (long long)XY * c);
                        const float wgt = w[0][a] * w[1][b] * w[2][c];
                        dens += (__ldg(mass + 4 * node) * wgt) * inv_cell_vol;
                    }
        }
        f[F_VOL * cap + i] = f[F_MASS * cap + i] / dens;
    }
}

// Scatter a live-order particle field back to the original order.
__global__ void gatherFieldKernel(const SceneDev* __restrict__ scenes, int scene, int parity, int field, int comps,
                                  int mode, float* __restrict__ out) {
    const SceneDev& sc = scenes[scene];
    const float* f = sc.buf[parity].f;
    const uint32_t* pid = sc.buf[parity].pid;
    const size_t cap = sc.cap;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads) {
        const uint32_t o = pid[i];
        if (mode == 1) {  // position4: one 16-byte store per particle
            reinterpret_cast<float4*>(out)[o] =
                make_float4(f[F_X * cap + i], f[(F_X + 1) * cap + i], f[(F_X + 2) * cap + i], 1.0f);
        } else if (mode == 2) {  // det of a 3x3 field
            float M[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) M[k] = f[(field + k) * cap + i];
            out[o] = det3(M);
        } else {
            for (int c = 0; c < comps; ++c) out[(size_t)comps * o + c] = f[(field + c) * cap + i];
        }
    }
}

// Overwrite a live-order particle field from original-order data.
__global__ void scatterFieldKernel(const SceneDev* __restrict__ scenes, int scene, int parity, int field, int comps,
                                   const float* __restrict__ in) {
    const SceneDev& sc = scenes[scene];
    float* f = sc.buf[parity].f;
    const uint32_t* pid = sc.buf[parity].pid;
    const size_t cap = sc.cap;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads) {
        const uint32_t o = pid[i];
        for (int c = 0; c < comps; ++c) f[(field + c) * cap + i] = in[(size_t)comps * o + c];
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers (host).
// ---------------------------------------------------------------------------
void launchKeys(const LaunchCtx& c, int parity, uint32_t* keys, uint32_t* block_count, uint32_t* err) {
    noteLaunches(1);
    keyKernel<<<dim3(c.particle_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes, parity, keys, block_count, err);
}

size_t compactScratchWords64(uint32_t total_blocks) {
    return (size_t)(total_blocks + kCompactTile - 1) / kCompactTile + 1;  // + the tile counter
}

void launchCompactOnesweep(const LaunchCtx& c, const BlockBuffers& bb, uint32_t total_blocks,
                           unsigned long long* scratch, uint32_t chunk, const ComboSplit& split, uint32_t* err) {
    const uint32_t ntiles = (uint32_t)((total_blocks + kCompactTile - 1) / kCompactTile);
    ClearRanges cr;
    cr.p[0] = reinterpret_cast<uint32_t*>(scratch);
    cr.n[0] = 2 * compactScratchWords64(total_blocks);
    cr.p[1] = bb.counters;
    cr.n[1] = 4;
    cr.p[2] = bb.counters + kG2PCountWord;
    cr.n[2] = kMaxCombos;
    cr.p[3] = bb.counters + kP2GListWord;  // lists, small, back
    cr.n[3] = 4 * kMaxCombos;
    launchClear(cr, c.stream);
    noteLaunches(1);
    compactOnesweepKernel<<<ntiles, kThreads, 0, c.stream>>>(
        bb.block_count, total_blocks, bb.scene_block_base, c.nscenes, bb.active, bb.outside, bb.counters,
        bb.block_slot, scratch + 1, reinterpret_cast<uint32_t*>(scratch), ntiles, chunk, bb.g2p_items, bb.g2p_cap,
        split, bb.p2g_lists, bb.p2g_list_cap, c.scenes, err);
}

void launchStress(const LaunchCtx& c, int parity) {
    noteLaunches(1);
    stressKernel<<<dim3(c.particle_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes, parity);
}

template <int S, int MODE, int STAGE>
static void setP2GAttr() {
    static bool done = false;
    if (!done) {
        cudaFuncSetAttribute(p2gKernel<S, MODE, STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)P2GLayout<S, MODE, STAGE>::smemBytes);
        done = true;
    }
}

// Particles staged per warp pass in P2G (16, 24 or 32): the engine's setting
// (mpm_tuning.p2g_stage, or its choice from the particle density).  Every
// size gives bitwise the same sums.
template <int S, int MODE, int STAGE>
static void p2gLaunch(const LaunchCtx& c, const StepArgs& a, int want) {
    setP2GAttr<S, MODE, STAGE>();
    p2gKernel<S, MODE, STAGE><<<c.persistent_blocks, P2GLayout<S, MODE, STAGE>::NT, P2GLayout<S, MODE, STAGE>::smemBytes,
                                c.stream>>>(a, want);
}

template <int S, int MODE>
static void p2gOne(const LaunchCtx& c, const StepArgs& a, int want) {
    switch (c.p2g_stage) {
        case 16: p2gLaunch<S, MODE, 16>(c, a, want); break;
        case 24: p2gLaunch<S, MODE, 24>(c, a, want); break;
        default: p2gLaunch<S, MODE, 32>(c, a, want); break;
    }
}

template <int S, int MODE>
static void p2gWarpLaunch(const LaunchCtx& c, const StepArgs& a) {
    using W = P2GWarpLayout<S, MODE>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(p2gWarpKernel<S, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)W::smemBytes);
        attr = true;
    }
    const unsigned grid = std::min<unsigned>(c.persistent_blocks, (unsigned)std::max(1, c.num_sms) * W::MIN_CTAS);
    p2gWarpKernel<S, MODE><<<grid, W::NT, W::smemBytes, c.stream>>>(a);
}

void launchP2GWarp(const LaunchCtx& c, const StepArgs& a, int S, int mode) {
    noteLaunches(1);
    const bool apic = mode == MODE_APIC_FUSED;
    if (S == 4) apic ? p2gWarpLaunch<4, MODE_APIC_FUSED>(c, a) : p2gWarpLaunch<4, MODE_FLIP>(c, a);
    else if (S == 3) apic ? p2gWarpLaunch<3, MODE_APIC_FUSED>(c, a) : p2gWarpLaunch<3, MODE_FLIP>(c, a);
    else apic ? p2gWarpLaunch<2, MODE_APIC_FUSED>(c, a) : p2gWarpLaunch<2, MODE_FLIP>(c, a);
}

void launchP2G(const LaunchCtx& c, const StepArgs& a, int S, int mode, int want_transfer) {
    noteLaunches(1);
#define P2G_CASE(SS)                                                                   \
    if (S == SS) {                                                                     \
        switch (mode) {                                                                \
            case MODE_APIC_FUSED: p2gOne<SS, MODE_APIC_FUSED>(c, a, want_transfer); break; \
            case MODE_FLIP: p2gOne<SS, MODE_FLIP>(c, a, want_transfer); break;         \
            case MODE_SPLIT: p2gOne<SS, MODE_SPLIT>(c, a, want_transfer); break;       \
            default: p2gOne<SS, MODE_MASS>(c, a, want_transfer); break;                \
        }                                                                              \
    }
    P2G_CASE(2) P2G_CASE(3) P2G_CASE(4)
#undef P2G_CASE
}

void launchGrid(const LaunchCtx& c, const StepArgs& a, int S, int mode, int want_transfer) {
    noteLaunches(1);
#define GRID_CASE(SS)                                                                                         \
    if (S == SS) {                                                                                            \
        switch (mode) {                                                                                       \
            case MODE_APIC_FUSED: gridKernel<SS, MODE_APIC_FUSED><<<c.persistent_blocks, kThreads, 0, c.stream>>>(a, want_transfer); break; \
            case MODE_FLIP: gridKernel<SS, MODE_FLIP><<<c.persistent_blocks, kThreads, 0, c.stream>>>(a, want_transfer); break; \
            case MODE_SPLIT: gridKernel<SS, MODE_SPLIT><<<c.persistent_blocks, kThreads, 0, c.stream>>>(a, want_transfer); break; \
            default: gridKernel<SS, MODE_MASS><<<c.persistent_blocks, kThreads, 0, c.stream>>>(a, want_transfer); break; \
        }                                                                                                     \
    }
    GRID_CASE(2) GRID_CASE(3) GRID_CASE(4)
#undef GRID_CASE
}

constexpr size_t kG2PDynSmem = sizeof(float) * 2 * kG2PThreads * kPreStride;
template <int S, bool APIC>
static void g2pLaunch(const LaunchCtx& c, const StepArgs& a, int fused) {
    static bool attr = [] {
        cudaFuncSetAttribute(g2pKernel<S, APIC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kG2PDynSmem);
        return true;
    }();
    (void)attr;
    g2pKernel<S, APIC><<<c.persistent_blocks * (256 / kG2PThreads), kG2PThreads, kG2PDynSmem, c.stream>>>(a, fused);
}

void launchG2P(const LaunchCtx& c, const StepArgs& args, int S, bool apic, bool fused, int combo) {
    noteLaunches(1);
    StepArgs a = args;
    a.combo = combo;
#define G2P_CASE(SS)                                  \
    if (S == SS) {                                    \
        if (apic) g2pLaunch<SS, true>(c, a, fused ? 1 : 0); \
        else g2pLaunch<SS, false>(c, a, fused ? 1 : 0);     \
    }
    G2P_CASE(2) G2P_CASE(3) G2P_CASE(4)
#undef G2P_CASE
}

void launchDenseGravity(const LaunchCtx& c) {
    noteLaunches(1);
    denseGravityKernel<<<dim3(c.node_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes);
}
void launchDenseUpdate(const LaunchCtx& c, float dt) {
    noteLaunches(1);
    denseUpdateVelocityKernel<<<dim3(c.node_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes, dt);
}
void launchDenseCollision(const LaunchCtx& c, float dt) {
    noteLaunches(1);
    denseCollisionKernel<<<dim3(c.node_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes, dt);
}
void launchDensePack(const LaunchCtx& c) {
    noteLaunches(1);
    densePackKernel<<<dim3(c.node_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes);
}
void launchParticlesCollision(const LaunchCtx& c, int parity, float dt) {
    noteLaunches(1);
    particlesCollisionKernel<<<dim3(c.particle_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes, parity, dt);
}
void launchAdvect(const LaunchCtx& c, int parity, float dt) {
    noteLaunches(1);
    advectKernel<<<dim3(c.particle_blocks, c.nscenes), kThreads, 0, c.stream>>>(c.scenes, parity, dt);
}
void launchInitState(cudaStream_t st, int num_sms, float* f, uint32_t* pid, uint16_t* mat, size_t cap,
                     const float* staged, size_t n, bool has_volume, const uint32_t* perm, const uint16_t* mat_in) {
    if (n == 0) return;
    noteLaunches(1);
    const unsigned blocks = (unsigned)std::min<size_t>((n + kThreads - 1) / kThreads, (size_t)num_sms * 8);
    initStateKernel<<<blocks, kThreads, 0, st>>>(f, pid, mat, cap, staged, n, has_volume ? 1 : 0, perm, mat_in);
}
void launchStagedKeys(cudaStream_t st, int num_sms, const SceneDev& sc, const float* xyz, uint32_t n, uint32_t* keys,
                      uint32_t* err) {
    if (n == 0) return;
    noteLaunches(1);
    const unsigned blocks = (unsigned)std::min<size_t>((n + kThreads - 1) / kThreads, (size_t)num_sms * 8);
    stagedKeyKernel<<<blocks, kThreads, 0, st>>>(sc, xyz, n, keys, err);
}
void launchVolume(const LaunchCtx& c, int parity, int S) {
    noteLaunches(1);
    dim3 g(c.particle_blocks, c.nscenes);
    if (S == 2) volumeKernel<2><<<g, kThreads, 0, c.stream>>>(c.scenes, parity);
    else if (S == 3) volumeKernel<3><<<g, kThreads, 0, c.stream>>>(c.scenes, parity);
    else volumeKernel<4><<<g, kThreads, 0, c.stream>>>(c.scenes, parity);
}
// Density rasterisation (writeToOpenVDB, src/mpm_solver3d.cu:509-572): node
// density = sum_p m_p w_ip / h^3, from the node masses of a mass pass.
__global__ void densityKernel(const float4* __restrict__ vstar, size_t nodes, float inv_cell_vol,
                              float* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)kThreads + threadIdx.x; i < nodes; i += (size_t)gridDim.x * kThreads)
        out[i] = vstar[i].w * inv_cell_vol;
}
// CFL time step (listed as unimplemented in the reference, README.md:60-67).
// A non-finite speed (NaN or Inf velocity, or |v|^2 overflowing) would leave
// dt without a bound (fmaxf drops NaN) or make it 0 (Inf): it raises
// ERR_NONFINITE, which the next synchronize reports as MPM_ERR_NUMERIC, and is
// left out of the maximum.
__global__ void __launch_bounds__(kThreads) cflMaxKernel(const SceneDev* __restrict__ scenes, int parity,
                                                         uint32_t* __restrict__ err) {
    const SceneDev& sc = scenes[blockIdx.y];
    if (!(sc.cfl > 0.f)) return;
    const float* f = sc.buf[parity].f;
    const size_t cap = sc.cap;
    float m = 0.f;
    bool bad = false;
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < sc.n; i += gridDim.x * kThreads) {
        const float vx = f[(F_V + 0) * cap + i], vy = f[(F_V + 1) * cap + i], vz = f[(F_V + 2) * cap + i];
        const float v2 = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
        if (isfinite(v2)) m = fmaxf(m, v2);
        else bad = true;
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(err, ERR_NONFINITE);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float wm[kThreads / 32];
    if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) m = fmaxf(m, wm[w]);
        if (m > 0.f) atomicMax(&sc.cfl_state->vmax2_bits, __float_as_uint(m));
    }
}
// One thread per scene: dt from the maximum, written into the (device) scene
// table that the step's kernels read, then the maximum is cleared.
__global__ void cflFinalizeKernel(SceneDev* __restrict__ scenes, int nscenes) {
    for (int i = threadIdx.x; i < nscenes; i += blockDim.x) {
        SceneDev& sc = scenes[i];
        if (!(sc.cfl > 0.f)) continue;
        CflState* st = sc.cfl_state;
        const float vmax = sqrtf(__uint_as_float(st->vmax2_bits));
        float dt = sc.dt_max;
        if (vmax > 0.f) dt = fminf(dt, __fdiv_rn(__fmul_rn(sc.cfl, sc.h), vmax));
        sc.dt = dt;
        st->vmax2_bits = 0u;
        st->last_dt = dt;
        st->time += (double)dt;
    }
}
void launchCfl(const LaunchCtx& c, int parity, size_t max_n, uint32_t* err) {
    noteLaunches(2);
    const unsigned bx = (unsigned)std::max<size_t>(
        1, std::min<size_t>((max_n + kThreads - 1) / kThreads, (size_t)c.num_sms * 4));
    cflMaxKernel<<<dim3(bx, (unsigned)c.nscenes), kThreads, 0, c.stream>>>(c.scenes, parity, err);
    cflFinalizeKernel<<<1, 128, 0, c.stream>>>(const_cast<SceneDev*>(c.scenes), c.nscenes);
}
void launchDensity(const LaunchCtx& c, const float4* vstar, size_t nodes, float inv_cell_vol, float* out) {
    noteLaunches(1);
    const unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((nodes + kThreads - 1) / kThreads,
                                                                          (size_t)c.num_sms * 16));
    densityKernel<<<blocks, kThreads, 0, c.stream>>>(vstar, nodes, inv_cell_vol, out);
}
// Loads the kernels of the host transfers (gather for downloads, scatter
// for uploads) on the current device: with CUDA's lazy loading a kernel is
// loaded at its first launch, which would otherwise stall a user's first
// download after the steps (about 2 ms).  Called once per device.
void preloadTransferKernels() {
    cudaFuncAttributes attr;
    cudaFuncGetAttributes(&attr, gatherFieldKernel);
    cudaFuncGetAttributes(&attr, scatterFieldKernel);
    cudaGetLastError();
}

void launchGatherField(const LaunchCtx& c, int scene, int parity, int field, int comps, int mode, float* out) {
    noteLaunches(1);
    gatherFieldKernel<<<c.particle_blocks, kThreads, 0, c.stream>>>(c.scenes, scene, parity, field, comps, mode, out);
}
void launchScatterField(const LaunchCtx& c, int scene, int parity, int field, int comps, const float* in) {
    noteLaunches(1);
    scatterFieldKernel<<<c.particle_blocks, kThreads, 0, c.stream>>>(c.scenes, scene, parity, field, comps, in);
}

// TMA tensor map of a dense float4 grid of res[0] x res[1] x res[2] nodes
// (node index x + X (y + Y z)) as a 4-D FP32 tensor (component, x, y, z),
// box (4, T, T, T), zero fill outside the grid.  The encoder is the driver's
// cuTensorMapEncodeTiled, fetched once through the runtime.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encodeTiledFn() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiledFn) nullptr;
        }
        return (EncodeTiledFn)p;
    }();
    return fn;
}
const char* encodeGridTensorMap(void* map, const void* grid, const int* res, int T) {
    static_assert(sizeof(CUtensorMap) == kTensorMapBytes, "tensor map size");
    EncodeTiledFn fn = encodeTiledFn();
    if (!fn) return "cuTensorMapEncodeTiled is not available from the driver";
    if (((uintptr_t)grid & 15u) != 0) return "grid buffer not 16-byte aligned";
    const cuuint64_t dims[4] = {4, (cuuint64_t)res[0], (cuuint64_t)res[1], (cuuint64_t)res[2]};
    const cuuint64_t strides[3] = {16, 16ull * (cuuint64_t)res[0], 16ull * (cuuint64_t)res[0] * (cuuint64_t)res[1]};
    const cuuint32_t box[4] = {4, (cuuint32_t)T, (cuuint32_t)T, (cuuint32_t)T};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUresult r = fn(reinterpret_cast<CUtensorMap*>(map), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                          const_cast<void*>(grid), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? nullptr : "cuTensorMapEncodeTiled rejected the grid tensor map";
}

size_t p2gSmemBytes(int S, int mode) {
#define SM_CASE(SS)                                                          \
    if (S == SS) {                                                           \
        switch (mode) {                                                      \
            case MODE_APIC_FUSED: return P2GLayout<SS, MODE_APIC_FUSED>::smemBytes; \
            case MODE_FLIP: return P2GLayout<SS, MODE_FLIP>::smemBytes;       \
            case MODE_SPLIT: return P2GLayout<SS, MODE_SPLIT>::smemBytes;     \
            default: return P2GLayout<SS, MODE_MASS>::smemBytes;              \
        }                                                                    \
    }
    SM_CASE(2) SM_CASE(3) SM_CASE(4)
#undef SM_CASE
    return 0;
}

}  // namespace mpm
