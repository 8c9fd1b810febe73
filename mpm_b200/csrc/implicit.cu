// implicit.cu -- semi-implicit grid velocity update for sm_100a.
//
// The reference declares solveLinearSystem(dt) and leaves it empty
// (src/mpm_solver3d.cu:312-314; IntegrationType in include/enums.h:17-21).
// This follows Stomakhin et al. 2013 ("A material point method for snow
// simulation", section 9): (M + beta dt^2 H) v = M v*, H the Hessian of the
// elastic energy in the grid node positions, applied matrix-free,
//     H u = sum_p V0 (dP/dF : (sum_j u_j grad w_jp^T) Fe) Fe^T grad w_ip,
// and solved by conjugate residual preconditioned with the node masses.
//
//   cellRangeKernel    first and end sorted position of every cell key and
//                      of every 4^3 block of cells
//   solvePrepKernel    per sorted particle: Fe, its SVD, cofactor, J, ln J,
//                      V0 mu and V0 la (hardened), model; the offsets
//                      (x - (o + h base)) / h of its stencil
//   solveInitKernel    node masses (the transfer's), x0 = v*, the other
//                      vectors 0, |M v*|^2, list of the nodes with mass
//   solveGatherKernel  per particle: G = sum_j u_j grad w^T, T = V0 dP(G Fe) Fe^T
//   solveScatterKernel per listed node: h = sum_p T_p grad w_ip
//   solveResidualKernel, solveAzKernel, solveUpdateKernel, solveDirKernel
//                      the elementwise vector updates and dot products
//   solveFinalKernel   v* = x (and the grid collision again in the fused step)
//
// A node's sum h is formed by one warp: the lanes share out the
// particles of the S^3 cells around the node (flattened, in sorted order) and
// the lane sums meet in a fixed shuffle tree, so a node's value does not
// depend on which warp computes it.  Dot products come from the elementwise
// kernels as per-block FP64 partials over a fixed node partition, which every
// consumer block reduces in block order.  The solve is bitwise reproducible
// and a scene's result does not depend on its batch-mates.  Convergence
// (|r| <= tol |M v*|) is decided on the device; a scene that converged skips
// the remaining launches of the step.
#include <cuda_runtime.h>
#include <stdint.h>

#include <climits>
#include <type_traits>

#include "engine_host.hpp"
#include "mpm_math.cuh"
#include "particle_common.cuh"

namespace mpm {

namespace {

enum { VX = 0, VR = 1, VZ = 2, VP = 3, VAP = 4, VAZ = 5, VH = 6 };  // node vectors
enum { QRR = 0, QZAZ = 1, QAPQ = 2, QBB = 3 };                      // dot products
static_assert(VH + 1 == kSolveVectors, "node vector count");

static_assert(kSolveBlocks == 2 * kThreads, "partials are reduced two per thread");

struct SolveArgs {
    const SceneDev* scenes;
    const uint32_t* sorted_keys;
    const uint32_t* perm;
    const uint2* cell_range;
    const uint2* block_range;
    float4* pofs;  // per sorted particle: stencil offsets d0 (xyz)
    float* prep;
    float4* T;
    uint32_t ntot;
    int parity;
    int split;
    int* iter;  // device iteration counter of the loop
};

// Prep planes (stride ntot): F 0..8, U 9..17, V 18..26, s 27..29, cof F
// 30..38, J 39, ln J 40, V0 mu 41, V0 la 42, model 43.
enum { PF = 0, PU = 9, PV = 18, PS = 27, PC = 30, PJ = 39, PLNJ = 40, PMU = 41, PLA = 42, PMODEL = 43 };
static_assert(PMODEL + 1 == kSolvePrepPlanes, "prep plane count");

__device__ __forceinline__ double* partSlot(const SceneDev& sc, int q, int j) {
    return sc.solve.part + ((size_t)q * (size_t)(sc.solve_max_iter + 2) + (size_t)j) * kSolveBlocks;
}

// Block-wide sum in a fixed order; the result is valid in every thread.
__device__ __forceinline__ double blockSum(double v) {
    __shared__ double sh[kThreads / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();  // sh may still be read by an earlier call
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += sh[w];
    return s;
}
// Sum of one slot's kSolveBlocks partials (same order in every block).
__device__ __forceinline__ double sumPartials(const double* p) {
    return blockSum(p[threadIdx.x] + p[threadIdx.x + kThreads]);
}
__device__ __forceinline__ void writePartial(double v, double* slot) {
    const double s = blockSum(v);
    if (threadIdx.x == 0) slot[blockIdx.x] = s;
}

__device__ __forceinline__ bool solving(const SceneDev& sc) { return sc.beta > 0.f; }
// The iteration at which the scene's solve converged, read once per block:
// the update kernel writes it while its other blocks read it, and every
// thread of a block must take the same branch before the block-wide sums.
__device__ __forceinline__ int blockDoneAt(const SceneDev& sc) {
    __shared__ int d;
    if (threadIdx.x == 0) d = sc.solve.status->done_at;
    __syncthreads();
    return d;
}
__device__ __forceinline__ size_t sceneNodes(const SceneDev& sc) {
    return (size_t)sc.res[0] * sc.res[1] * sc.res[2];
}
__device__ __forceinline__ void nodeCoords(const SceneDev& sc, size_t node, int* n) {
    n[0] = (int)(node % (size_t)sc.res[0]);
    n[1] = (int)((node / (size_t)sc.res[0]) % (size_t)sc.res[1]);
    n[2] = (int)(node / ((size_t)sc.res[0] * sc.res[1]));
}
__device__ __forceinline__ float3 ld3(const float4& v) { return make_float3(v.x, v.y, v.z); }

// Weight and gradient of stencil node k of a particle with stencil offsets
// d0 = (x - (o + h base)) / h (the distance is d0 - k, as in G2P).
template <int S>
__device__ __forceinline__ void nodeWeight(const SceneDev& sc, const float4& d0, const int* k, float* w, float* dw) {
    const float d[3] = {d0.x - (float)k[0], d0.y - (float)k[1], d0.z - (float)k[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        w[a] = splineN<S>(d[a]);
        dw[a] = splineNDot<S>(d[a]) * sc.inv_h;
    }
}
// Stencil base of a particle from its cell key (key = block << 6 | cell,
// base + 4 = 4 block + cell per axis).
__device__ __forceinline__ void keyBase(const SceneDev& sc, uint32_t key, int* base) {
    const uint32_t lb = (key >> 6) - sc.block_base, c = key & 63u;
    base[0] = 4 * (int)(lb % (uint32_t)sc.nb[0]) - 4 + (int)(c & 3u);
    base[1] = 4 * (int)((lb / (uint32_t)sc.nb[0]) % (uint32_t)sc.nb[1]) - 4 + (int)((c >> 2) & 3u);
    base[2] = 4 * (int)(lb / ((uint32_t)sc.nb[0] * sc.nb[1])) - 4 + (int)(c >> 4);
}

// Sum fn(p, base, k) over the particles whose stencil covers node n, by one
// warp: the S^3 base cells n - S + 1 .. n (always inside the key range) in a
// fixed order, their particles in sorted order, flattened and dealt to the
// lanes round-robin; the lane sums meet in a fixed shuffle tree.  Every lane
// returns the total.  sh: this warp's 2 S^3 + 1 ints of shared memory.
template <int S, int C, class Fn>
__device__ __forceinline__ void warpNodeSum(const SceneDev& sc, const SolveArgs& a, const int* n, int* sh, float* out,
                                            Fn&& fn) {
    constexpr int NC = S * S * S;
    const int lane = threadIdx.x & 31;
    int* first = sh;       // NC
    int* start = sh + NC;  // NC + 1: flattened offset of each cell
    int cnt[2] = {0, 0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int ci = lane + 32 * h;
        if (ci < NC) {
            const int c[3] = {ci % S, (ci / S) % S, ci / (S * S)};
            const int base[3] = {n[0] - S + 1 + c[0], n[1] - S + 1 + c[1], n[2] - S + 1 + c[2]};
            const uint2 rg = a.cell_range[makeKey(sc, base)];
            first[ci] = (int)rg.x;
            cnt[h] = (int)(rg.y - rg.x);
        }
    }
    // exclusive offsets in cell order: cells lane and 32 + lane
    int v0 = cnt[0], v1 = cnt[1];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t0 = __shfl_up_sync(0xffffffffu, v0, o), t1 = __shfl_up_sync(0xffffffffu, v1, o);
        if (lane >= o) {
            v0 += t0;
            v1 += t1;
        }
    }
    const int tot0 = __shfl_sync(0xffffffffu, v0, 31);
    if (lane < NC) start[lane] = v0 - cnt[0];
    if (32 + lane < NC) start[32 + lane] = tot0 + v1 - cnt[1];
    const int total = tot0 + __shfl_sync(0xffffffffu, v1, 31);
    if (lane == 0) start[NC] = total;
    __syncwarp();
    float acc[C];
#pragma unroll
    for (int q = 0; q < C; ++q) acc[q] = 0.f;
    for (int f = lane; f < total; f += 32) {
        int lo = 0, hi = NC - 1;  // the cell with start[ci] <= f < start[ci + 1]
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (start[mid] <= f) lo = mid;
            else hi = mid - 1;
        }
        const int c[3] = {lo % S, (lo / S) % S, lo / (S * S)};
        const int base[3] = {n[0] - S + 1 + c[0], n[1] - S + 1 + c[1], n[2] - S + 1 + c[2]};
        const int k[3] = {S - 1 - c[0], S - 1 - c[1], S - 1 - c[2]};
        fn((uint32_t)(first[lo] + (f - start[lo])), base, k, acc);
    }
#pragma unroll
    for (int q = 0; q < C; ++q) {
        float v = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        out[q] = __shfl_sync(0xffffffffu, v, 0);  // lane 0's tree order
    }
    __syncwarp();  // sh is reused by the warp's next node
}

__device__ __forceinline__ void ldMat(const float* prep, size_t stride, size_t i, int plane, float* m) {
#pragma unroll
    for (int e = 0; e < 9; ++e) m[e] = prep[(size_t)(plane + e) * stride + i];
}
__device__ __forceinline__ void cross3(const float* a, const float* b, float* c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
// Cofactor J F^-T by columns (c_k = f_{k+1} x f_{k+2}), row-major.
__device__ __forceinline__ void cofactor(const float* F, float* C) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int a = (k + 1) % 3, b = (k + 2) % 3;
        const float fa[3] = {F[a], F[3 + a], F[6 + a]}, fb[3] = {F[b], F[3 + b], F[6 + b]};
        float c[3];
        cross3(fa, fb, c);
#pragma unroll
        for (int r = 0; r < 3; ++r) C[3 * r + k] = c[r];
    }
}
__device__ __forceinline__ void cofactorDifferential(const float* F, const float* dF, float* dC) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int a = (k + 1) % 3, b = (k + 2) % 3;
        const float da[3] = {dF[a], dF[3 + a], dF[6 + a]}, fb[3] = {F[b], F[3 + b], F[6 + b]};
        const float fa[3] = {F[a], F[3 + a], F[6 + a]}, db[3] = {dF[b], dF[3 + b], dF[6 + b]};
        float c1[3], c2[3];
        cross3(da, fb, c1);
        cross3(fa, db, c2);
#pragma unroll
        for (int r = 0; r < 3; ++r) dC[3 * r + k] = c1[r] + c2[r];
    }
}
__device__ __forceinline__ void mm3(const float* A, const float* B, float* C) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[3 * i] * B[j] + A[3 * i + 1] * B[3 + j] + A[3 * i + 2] * B[6 + j];
}
__device__ __forceinline__ void mm3T(const float* A, const float* B, float* C) {  // A B^T
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            C[3 * i + j] = A[3 * i] * B[3 * j] + A[3 * i + 1] * B[3 * j + 1] + A[3 * i + 2] * B[3 * j + 2];
}
__device__ __forceinline__ void mTm3(const float* A, const float* B, float* C) {  // A^T B
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[3 * i + j] = A[i] * B[j] + A[3 + i] * B[3 + j] + A[6 + i] * B[6 + j];
}

}  // namespace

// ---------------------------------------------------------------------------
__global__ void cellRangeKernel(const uint32_t* __restrict__ keys, uint32_t n, uint2* __restrict__ range,
                                uint2* __restrict__ block_range) {
    for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const uint32_t k = keys[i];
        const uint32_t kp = i > 0 ? keys[i - 1] : 0xffffffffu, kn = i + 1 < n ? keys[i + 1] : 0xffffffffu;
        if (kp != k) range[k].x = i;
        if (kn != k) range[k].y = i + 1;
        if (i == 0 || (kp >> 6) != (k >> 6)) block_range[k >> 6].x = i;
        if (i + 1 == n || (kn >> 6) != (k >> 6)) block_range[k >> 6].y = i + 1;
    }
}

__global__ void __launch_bounds__(kThreads) solvePrepKernel(SolveArgs a) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    if (!solving(sc)) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) *sc.solve.status = SolveStatus{INT_MAX, 0, 0.f, 0};
    const float* f = sc.buf[a.parity].f;
    const uint16_t* mat = sc.buf[a.parity].mat;
    const size_t cap = sc.cap, st = a.ntot;
    for (uint32_t j = blockIdx.x * kThreads + threadIdx.x; j < sc.n; j += gridDim.x * kThreads) {
        const size_t i = (size_t)sc.key_offset + j;
        const uint32_t slot = a.perm[i] - sc.key_offset;
        float F[9], Fp[9], U[9], V[9], s[3], C[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            F[e] = f[(size_t)(F_FE + e) * cap + slot];
            Fp[e] = f[(size_t)(F_FP + e) * cap + slot];
        }
        // material ids are kept (and copied between the buffers) only for
        // scenes with several materials
        const MaterialDev md = sc.mats[sc.nmat > 1 ? mat[slot] : 0];
        float mu, la;
        plasticLame(md, Fp, mu, la);
        const float V0 = f[(size_t)F_VOL * cap + slot];
        svd3(F, U, s, V);
        cofactor(F, C);
        const float J = det3(F);
        float* p = a.prep + i;
#pragma unroll
        for (int e = 0; e < 9; ++e) {
            p[(size_t)(PF + e) * st] = F[e];
            p[(size_t)(PU + e) * st] = U[e];
            p[(size_t)(PV + e) * st] = V[e];
            p[(size_t)(PC + e) * st] = C[e];
        }
#pragma unroll
        for (int e = 0; e < 3; ++e) p[(size_t)(PS + e) * st] = s[e];
        p[(size_t)PJ * st] = J;
        p[(size_t)PLNJ * st] = md.model == MPM_MODEL_NEO_HOOKEAN ? logf(J) : 0.f;
        p[(size_t)PMU * st] = V0 * mu;
        p[(size_t)PLA * st] = V0 * la;
        p[(size_t)PMODEL * st] = (float)md.model;
        const float x[3] = {f[(size_t)(F_X + 0) * cap + slot], f[(size_t)(F_X + 1) * cap + slot],
                            f[(size_t)(F_X + 2) * cap + slot]};
        int base[3];
        float d0[3] = {0.f, 0.f, 0.f};
        if (stencilBase(sc, x, base)) {  // else an outside particle: no stencil
#pragma unroll
            for (int ax = 0; ax < 3; ++ax)
                d0[ax] = __fdiv_rn(x[ax] - __fadd_rn(sc.origin[ax], __fmul_rn(sc.h, (float)base[ax])), sc.h);
        }
        a.pofs[i] = make_float4(d0[0], d0[1], d0[2], 0.f);
    }
}

// Node masses, x0 = v*, the other vectors 0, |M v*|^2, and the list of the
// nodes with mass.  The masses are the transfer's own: the split-mode grid
// holds them densely; in the fused step the grid pass wrote (v*, m) for the
// node blocks N (nodes 4N - 4 + L) next to a particle block N - (0|1, 0|1,
// 0|1) that holds particles, and the other nodes have no mass this step.
__global__ void __launch_bounds__(kThreads) solveInitKernel(SolveArgs a) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    if (!solving(sc)) return;
    const size_t nodes = sceneNodes(sc);
    float4* vec = sc.solve.vec;
    double acc = 0.0;
    for (size_t node = (size_t)blockIdx.x * kThreads + threadIdx.x; node < nodes;
         node += (size_t)kSolveBlocks * kThreads) {
        float m = 0.f, vs[3] = {0.f, 0.f, 0.f};
        if (a.split) {
            m = sc.dbg[node];
#pragma unroll
            for (int c = 0; c < 3; ++c) vs[c] = sc.dbg[(size_t)(7 + c) * nodes + node];
        } else {
            int n[3];
            nodeCoords(sc, node, n);
            const int N[3] = {(n[0] + 4) >> 2, (n[1] + 4) >> 2, (n[2] + 4) >> 2};
            bool written = false;
#pragma unroll
            for (int d = 0; d < 8; ++d) {
                const int B[3] = {N[0] - (d & 1), N[1] - ((d >> 1) & 1), N[2] - (d >> 2)};
                if (B[0] >= 0 && B[1] >= 0 && B[2] >= 0 && B[0] < sc.nb[0] && B[1] < sc.nb[1] && B[2] < sc.nb[2]) {
                    const uint2 r = a.block_range[sc.block_base + (uint32_t)((B[2] * sc.nb[1] + B[1]) * sc.nb[0] + B[0])];
                    written |= r.y > r.x;
                }
            }
            if (written) {
                const float4 v = sc.vstar[node];
                m = v.w;
                vs[0] = v.x;
                vs[1] = v.y;
                vs[2] = v.z;
            }
        }
        const bool act = m > kFltEps;
        if (act) {
            acc += (double)(m * vs[0]) * (m * vs[0]) + (double)(m * vs[1]) * (m * vs[1]) +
                   (double)(m * vs[2]) * (m * vs[2]);
            sc.solve.list[atomicAdd(&sc.solve.status->nactive, 1)] = (int)node;
        }
        sc.solve.m[node] = act ? m : 0.f;
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        vec[(size_t)VX * nodes + node] = act ? make_float4(vs[0], vs[1], vs[2], 0.f) : z4;
#pragma unroll
        for (int v = VR; v <= VH; ++v) vec[(size_t)v * nodes + node] = z4;
    }
    writePartial(acc, partSlot(sc, QBB, 0));
}

template <int S>
__global__ void __launch_bounds__(kThreads) solveGatherKernel(SolveArgs a, int src, const int* kp, int k0) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    const int k = kp ? *kp : k0;
    if (!solving(sc) || sc.S != S || blockDoneAt(sc) <= k) return;
    const size_t nodes = sceneNodes(sc), st = a.ntot;
    const float4* u = sc.solve.vec + (size_t)src * nodes;
    const uint32_t outside = sc.block_base + sc.nblocks;
    for (uint32_t j = blockIdx.x * kThreads + threadIdx.x; j < sc.n; j += gridDim.x * kThreads) {
        const size_t i = (size_t)sc.key_offset + j;
        float4* To = a.T + 3 * i;
        const uint32_t key = a.sorted_keys[i];
        if ((key >> 6) >= outside) {
            To[0] = To[1] = To[2] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        int base[3];
        keyBase(sc, key, base);
        const float4 q = a.pofs[i];
        const float d0[3] = {q.x, q.y, q.z};
        float w[3][S], dw[3][S];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            float dk[S];
            dk[0] = d0[ax];
#pragma unroll
            for (int kk = 1; kk < S; ++kk) dk[kk] = dk[0] - (float)kk;
            splineWeights<S>(dk, w[ax], dw[ax]);
#pragma unroll
            for (int kk = 0; kk < S; ++kk) dw[ax][kk] *= sc.inv_h;
        }
        float G[9];
#pragma unroll
        for (int e = 0; e < 9; ++e) G[e] = 0.f;
#pragma unroll
        for (int c = 0; c < S; ++c) {
            const int nz = base[2] + c;
            if (nz < 0 || nz >= sc.res[2]) continue;
#pragma unroll
            for (int b = 0; b < S; ++b) {
                const int ny = base[1] + b;
                if (ny < 0 || ny >= sc.res[1]) continue;
#pragma unroll
                for (int ai = 0; ai < S; ++ai) {
                    const int nx = base[0] + ai;
                    if (nx < 0 || nx >= sc.res[0]) continue;
                    const float3 uv = ld3(u[(size_t)nx + (size_t)sc.res[0] * ((size_t)ny + (size_t)sc.res[1] * nz)]);
                    const float g[3] = {dw[0][ai] * w[1][b] * w[2][c], w[0][ai] * dw[1][b] * w[2][c],
                                        w[0][ai] * w[1][b] * dw[2][c]};
#pragma unroll
                    for (int col = 0; col < 3; ++col) {
                        G[col] += uv.x * g[col];
                        G[3 + col] += uv.y * g[col];
                        G[6 + col] += uv.z * g[col];
                    }
                }
            }
        }
        float F[9], C[9], dF[9], dP[9];
        ldMat(a.prep, st, i, PF, F);
        ldMat(a.prep, st, i, PC, C);
        mm3(G, F, dF);
        const float vmu = a.prep[(size_t)PMU * st + i], vla = a.prep[(size_t)PLA * st + i];
        const float J = a.prep[(size_t)PJ * st + i];
        float dJ = 0.f;
#pragma unroll
        for (int e = 0; e < 9; ++e) dJ += C[e] * dF[e];
        if (a.prep[(size_t)PMODEL * st + i] == (float)MPM_MODEL_NEO_HOOKEAN) {
            // dP = mu dF - (la ln J - mu) F^-T dF^T F^-T + la (F^-T : dF) F^-T
            float FiT[9], tmp[9], dFiT[9];
            const float invJ = 1.0f / J;
#pragma unroll
            for (int e = 0; e < 9; ++e) FiT[e] = C[e] * invJ;
            mm3T(FiT, dF, tmp);   // F^-T dF^T
            mm3(tmp, FiT, dFiT);  // F^-T dF^T F^-T
            const float lnJ = a.prep[(size_t)PLNJ * st + i];
            const float dlnJ = dJ * invJ;
#pragma unroll
            for (int e = 0; e < 9; ++e) dP[e] = vmu * dF[e] - (vla * lnJ - vmu) * dFiT[e] + vla * dlnJ * FiT[e];
        } else {
            // dP = 2 mu (dF - dR) + la (dJ cof F + (J - 1) dcof F), dR = U W V^T
            float U[9], V[9], M[9], tmp[9], W[9], dR[9], dC[9];
            ldMat(a.prep, st, i, PU, U);
            ldMat(a.prep, st, i, PV, V);
            const float s0 = a.prep[(size_t)(PS + 0) * st + i], s1 = a.prep[(size_t)(PS + 1) * st + i],
                        s2 = a.prep[(size_t)(PS + 2) * st + i];
            mTm3(U, dF, tmp);  // U^T dF
            mm3(tmp, V, M);    // U^T dF V
            auto den = [](float d) { return fabsf(d) < 1e-6f ? (d < 0.f ? -1e-6f : 1e-6f) : d; };
            const float w01 = (M[1] - M[3]) / den(s0 + s1), w02 = (M[2] - M[6]) / den(s0 + s2),
                        w12 = (M[5] - M[7]) / den(s1 + s2);
            W[0] = 0.f, W[1] = w01, W[2] = w02;
            W[3] = -w01, W[4] = 0.f, W[5] = w12;
            W[6] = -w02, W[7] = -w12, W[8] = 0.f;
            mm3(U, W, tmp);
            mm3T(tmp, V, dR);
            cofactorDifferential(F, dF, dC);
#pragma unroll
            for (int e = 0; e < 9; ++e) dP[e] = 2.0f * vmu * (dF[e] - dR[e]) + vla * (dJ * C[e] + (J - 1.0f) * dC[e]);
        }
        float Tm[9];
        mm3T(dP, F, Tm);  // V0 dP Fe^T
        To[0] = make_float4(Tm[0], Tm[1], Tm[2], 0.f);
        To[1] = make_float4(Tm[3], Tm[4], Tm[5], 0.f);
        To[2] = make_float4(Tm[6], Tm[7], Tm[8], 0.f);
    }
}

// h = sum_p T_p grad w_ip at the listed nodes (one warp per node).
template <int S>
__global__ void __launch_bounds__(kThreads) solveScatterKernel(SolveArgs a, const int* kp, int k0) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    const int k = kp ? *kp : k0;
    if (!solving(sc) || sc.S != S || blockDoneAt(sc) <= k) return;
    __shared__ int sh[kThreads / 32][2 * S * S * S + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const size_t nodes = sceneNodes(sc);
    float4* h = sc.solve.vec + (size_t)VH * nodes;
    const int na = sc.solve.status->nactive;
    for (int li = blockIdx.x * (kThreads / 32) + warp; li < na; li += gridDim.x * (kThreads / 32)) {
        const size_t node = (size_t)sc.solve.list[li];
        int n[3];
        nodeCoords(sc, node, n);
        float out[3];
        warpNodeSum<S, 3>(sc, a, n, sh[warp], out, [&](uint32_t p, const int* base, const int* kk, float* acc) {
            float w[3], dw[3];
            nodeWeight<S>(sc, a.pofs[p], kk, w, dw);
            const float g[3] = {dw[0] * w[1] * w[2], w[0] * dw[1] * w[2], w[0] * w[1] * dw[2]};
            const float4* Tp = a.T + 3 * (size_t)p;
            const float4 t0 = Tp[0], t1 = Tp[1], t2 = Tp[2];
            acc[0] += t0.x * g[0] + t0.y * g[1] + t0.z * g[2];
            acc[1] += t1.x * g[0] + t1.y * g[1] + t1.z * g[2];
            acc[2] += t2.x * g[0] + t2.y * g[1] + t2.z * g[2];
        });
        if (lane == 0) h[node] = make_float4(out[0], out[1], out[2], 0.f);
    }
}

// x0 = v*: r0 = -c H v*, z0 = r0 / m, |r0|^2.
__global__ void __launch_bounds__(kThreads) solveResidualKernel(SolveArgs a) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    if (!solving(sc)) return;
    const size_t nodes = sceneNodes(sc);
    float4* vec = sc.solve.vec;
    const float c = sc.beta * sc.dt * sc.dt;
    double acc = 0.0;
    for (size_t node = (size_t)blockIdx.x * kThreads + threadIdx.x; node < nodes;
         node += (size_t)kSolveBlocks * kThreads) {
        const float m = sc.solve.m[node];
        if (!(m > 0.f)) continue;
        const float3 h = ld3(vec[(size_t)VH * nodes + node]);
        const float r[3] = {-c * h.x, -c * h.y, -c * h.z};
        vec[(size_t)VR * nodes + node] = make_float4(r[0], r[1], r[2], 0.f);
        vec[(size_t)VZ * nodes + node] = make_float4(r[0] / m, r[1] / m, r[2] / m, 0.f);
        acc += (double)r[0] * r[0] + (double)r[1] * r[1] + (double)r[2] * r[2];
    }
    writePartial(acc, partSlot(sc, QRR, 0));
}

// Az = M z + c H z, (z, Az) into slot j.
__global__ void __launch_bounds__(kThreads) solveAzKernel(SolveArgs a, const int* kp, int j0, int k0) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    const int k = kp ? *kp : k0, j = kp ? k + 1 : j0;
    if (!solving(sc) || blockDoneAt(sc) <= k) return;
    const size_t nodes = sceneNodes(sc);
    float4* vec = sc.solve.vec;
    const float c = sc.beta * sc.dt * sc.dt;
    double acc = 0.0;
    for (size_t node = (size_t)blockIdx.x * kThreads + threadIdx.x; node < nodes;
         node += (size_t)kSolveBlocks * kThreads) {
        const float m = sc.solve.m[node];
        if (!(m > 0.f)) continue;
        const float3 z = ld3(vec[(size_t)VZ * nodes + node]), h = ld3(vec[(size_t)VH * nodes + node]);
        const float Az[3] = {m * z.x + c * h.x, m * z.y + c * h.y, m * z.z + c * h.z};
        vec[(size_t)VAZ * nodes + node] = make_float4(Az[0], Az[1], Az[2], 0.f);
        acc += (double)z.x * Az[0] + (double)z.y * Az[1] + (double)z.z * Az[2];
    }
    writePartial(acc, partSlot(sc, QZAZ, j));
}

// p = z + gamma p, Ap = Az + gamma Ap (gamma = 0 at j = 0), partial (Ap, M^-1 Ap).
__global__ void __launch_bounds__(kThreads) solveDirKernel(SolveArgs a, const int* kp, int j0, int k0) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    const int k = kp ? *kp : k0, j = kp ? k + 1 : j0;
    if (!solving(sc) || blockDoneAt(sc) <= k) return;
    const size_t nodes = sceneNodes(sc);
    float4* vec = sc.solve.vec;
    float gam = 0.f;
    if (j > 0) gam = (float)(sumPartials(partSlot(sc, QZAZ, j)) / sumPartials(partSlot(sc, QZAZ, j - 1)));
    double acc = 0.0;
    for (size_t node = (size_t)blockIdx.x * kThreads + threadIdx.x; node < nodes;
         node += (size_t)kSolveBlocks * kThreads) {
        const float m = sc.solve.m[node];
        if (!(m > 0.f)) continue;
        const float3 z = ld3(vec[(size_t)VZ * nodes + node]), p = ld3(vec[(size_t)VP * nodes + node]);
        const float3 Az = ld3(vec[(size_t)VAZ * nodes + node]), Ap = ld3(vec[(size_t)VAP * nodes + node]);
        const float np[3] = {z.x + gam * p.x, z.y + gam * p.y, z.z + gam * p.z};
        const float nAp[3] = {Az.x + gam * Ap.x, Az.y + gam * Ap.y, Az.z + gam * Ap.z};
        vec[(size_t)VP * nodes + node] = make_float4(np[0], np[1], np[2], 0.f);
        vec[(size_t)VAP * nodes + node] = make_float4(nAp[0], nAp[1], nAp[2], 0.f);
        acc += ((double)nAp[0] * nAp[0] + (double)nAp[1] * nAp[1] + (double)nAp[2] * nAp[2]) / m;
    }
    writePartial(acc, partSlot(sc, QAPQ, j));
}

// Iteration k: convergence test, then x += alpha p, r -= alpha Ap, z -= alpha M^-1 Ap.
__global__ void __launch_bounds__(kThreads) solveUpdateKernel(SolveArgs a, const int* kp) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    const int k = *kp;
    if (!solving(sc) || blockDoneAt(sc) <= k) return;
    bool done = k >= sc.solve_max_iter;
    double zAz = 0.0, Apq = 0.0;
    if (!done) {
        const double rr = sumPartials(partSlot(sc, QRR, k)), bb = sumPartials(partSlot(sc, QBB, 0));
        zAz = sumPartials(partSlot(sc, QZAZ, k));
        Apq = sumPartials(partSlot(sc, QAPQ, k));
        const double tol = sc.solve_tol;
        done = rr <= tol * tol * bb || !(Apq > 0.0) || !isfinite(zAz);
    }
    if (done) {  // every block takes the same decision; block 0 records it
        if (blockIdx.x == 0 && threadIdx.x == 0) sc.solve.status->done_at = k;
        return;
    }
    const float alpha = (float)(zAz / Apq);
    const size_t nodes = sceneNodes(sc);
    float4* vec = sc.solve.vec;
    double acc = 0.0;
    for (size_t node = (size_t)blockIdx.x * kThreads + threadIdx.x; node < nodes;
         node += (size_t)kSolveBlocks * kThreads) {
        const float m = sc.solve.m[node];
        if (!(m > 0.f)) continue;
        const float3 x = ld3(vec[(size_t)VX * nodes + node]), r = ld3(vec[(size_t)VR * nodes + node]);
        const float3 z = ld3(vec[(size_t)VZ * nodes + node]), p = ld3(vec[(size_t)VP * nodes + node]);
        const float3 Ap = ld3(vec[(size_t)VAP * nodes + node]);
        const float nr[3] = {r.x - alpha * Ap.x, r.y - alpha * Ap.y, r.z - alpha * Ap.z};
        vec[(size_t)VX * nodes + node] = make_float4(x.x + alpha * p.x, x.y + alpha * p.y, x.z + alpha * p.z, 0.f);
        vec[(size_t)VR * nodes + node] = make_float4(nr[0], nr[1], nr[2], 0.f);
        vec[(size_t)VZ * nodes + node] =
            make_float4(z.x - alpha * (Ap.x / m), z.y - alpha * (Ap.y / m), z.z - alpha * (Ap.z / m), 0.f);
        acc += (double)nr[0] * nr[0] + (double)nr[1] * nr[1] + (double)nr[2] * nr[2];
    }
    writePartial(acc, partSlot(sc, QRR, k + 1));
}

// End of iteration k: is any scene still iterating (not converged by the
// test of iteration k, k + 1 < its max_iter)?  Advances the counter and, in a
// graph, sets the condition of the loop node.
__global__ void solveCondKernel(SolveArgs a, int nscenes, cudaGraphConditionalHandle h, int use_cond) {
    const int k = *a.iter;
    int running = 0;
    for (int i = threadIdx.x; i < nscenes; i += blockDim.x) {
        const SceneDev& sc = a.scenes[i];
        if (solving(sc) && sc.solve.status->done_at > k && k + 1 < sc.solve_max_iter) running = 1;
    }
    running = __syncthreads_or(running);
    if (threadIdx.x == 0) {
        *a.iter = k + 1;
        if (use_cond) cudaGraphSetConditional(h, running ? 1u : 0u);
    }
}

__global__ void __launch_bounds__(kThreads) solveFinalKernel(SolveArgs a) {
    const SceneDev& sc = a.scenes[blockIdx.y];
    if (!solving(sc)) return;
    const int done_at = blockDoneAt(sc);
    const int iters = done_at < sc.solve_max_iter ? done_at : sc.solve_max_iter;
    const double rr = sumPartials(partSlot(sc, QRR, iters)), bb = sumPartials(partSlot(sc, QBB, 0));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc.solve.status->iters = iters;
        sc.solve.status->residual = bb > 0.0 ? (float)sqrt(rr / bb) : 0.f;
    }
    const size_t nodes = sceneNodes(sc);
    for (size_t node = (size_t)blockIdx.x * kThreads + threadIdx.x; node < nodes;
         node += (size_t)kSolveBlocks * kThreads) {
        if (!(sc.solve.m[node] > 0.f)) continue;
        const float3 x = ld3(sc.solve.vec[(size_t)VX * nodes + node]);
        float vs[3] = {x.x, x.y, x.z};
        if (a.split) {
#pragma unroll
            for (int c = 0; c < 3; ++c) sc.dbg[(size_t)(7 + c) * nodes + node] = vs[c];
        } else {
            int n[3];
            nodeCoords(sc, node, n);
            gridNodeCollision(sc, n, sc.dt, vs);
            const float w = sc.vstar[node].w;
            sc.vstar[node] = make_float4(vs[0], vs[1], vs[2], w);
        }
    }
}

// ---------------------------------------------------------------------------
cudaError_t launchSolve(const LaunchCtx& c, const SolveBuffers& b, int parity, const int* stencils, int nstencils,
                        int max_iter, bool split, cudaStream_t aux) {
    SolveArgs a{c.scenes, b.sorted_keys, b.perm, b.cell_range, b.block_range, b.pofs, b.prep, b.T, b.ntot, parity,
                split ? 1 : 0, b.iter};
    const dim3 pgrid(c.particle_blocks, (unsigned)c.nscenes), ngrid(kSolveBlocks, (unsigned)c.nscenes);
    const dim3 wgrid((unsigned)c.num_sms * 8, (unsigned)c.nscenes);  // warp-per-node kernels
    uint64_t launches = 0;
    cudaMemsetAsync(b.cell_range, 0, sizeof(uint2) * b.nkeys, c.stream);
    cudaMemsetAsync(b.block_range, 0, sizeof(uint2) * b.nblocks, c.stream);
    const unsigned kb = (unsigned)std::max<size_t>(
        1, std::min<size_t>((b.ntot + kThreads - 1) / kThreads, (size_t)c.num_sms * 8));
    cellRangeKernel<<<kb, kThreads, 0, c.stream>>>(b.sorted_keys, b.ntot, b.cell_range, b.block_range);
    solvePrepKernel<<<pgrid, kThreads, 0, c.stream>>>(a);
    launches += 2;
    auto perS = [&](auto launch) {
        for (int i = 0; i < nstencils; ++i) {
            switch (stencils[i]) {
                case 2: launch(std::integral_constant<int, 2>{}); break;
                case 3: launch(std::integral_constant<int, 3>{}); break;
                default: launch(std::integral_constant<int, 4>{}); break;
            }
            ++launches;
        }
    };
    cudaStream_t st = c.stream;  // the stream of the iteration kernels
    const int* kp = nullptr;
    auto gatherX = [&](auto S) { solveGatherKernel<decltype(S)::value><<<pgrid, kThreads, 0, st>>>(a, VX, nullptr, -1); };
    auto gatherZ = [&](auto S) { solveGatherKernel<decltype(S)::value><<<pgrid, kThreads, 0, st>>>(a, VZ, kp, -1); };
    auto scatter = [&](auto S) { solveScatterKernel<decltype(S)::value><<<wgrid, kThreads, 0, st>>>(a, kp, -1); };
    solveInitKernel<<<ngrid, kThreads, 0, st>>>(a);
    perS(gatherX);
    perS(scatter);
    solveResidualKernel<<<ngrid, kThreads, 0, st>>>(a);
    perS(gatherZ);
    perS(scatter);
    solveAzKernel<<<ngrid, kThreads, 0, st>>>(a, nullptr, 0, -1);
    solveDirKernel<<<ngrid, kThreads, 0, st>>>(a, nullptr, 0, -1);
    cudaMemsetAsync(b.iter, 0, sizeof(int), st);
    launches += 4;
    kp = b.iter;
    auto body = [&](cudaGraphConditionalHandle h, int use_cond) {
        solveUpdateKernel<<<ngrid, kThreads, 0, st>>>(a, kp);
        perS(gatherZ);
        perS(scatter);
        solveAzKernel<<<ngrid, kThreads, 0, st>>>(a, kp, 0, 0);
        solveDirKernel<<<ngrid, kThreads, 0, st>>>(a, kp, 0, 0);
        solveCondKernel<<<1, kThreads, 0, st>>>(a, c.nscenes, h, use_cond);
        launches += 4;
    };
    // Inside a stream capture the iterations become a conditional while node
    // (the body captured once on the auxiliary stream), so a converged solve
    // launches nothing more; direct launches run max_iter bodies, whose
    // kernels return at once after convergence.
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(c.stream, &cs);
    if (e != cudaSuccess) return e;
    if (cs == cudaStreamCaptureStatusActive && aux) {
        cudaGraph_t g = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        if ((e = cudaStreamGetCaptureInfo(c.stream, &cs, nullptr, &g, &deps, &nd)) != cudaSuccess) return e;
        cudaGraphConditionalHandle h;
        if ((e = cudaGraphConditionalHandleCreate(&h, g, 1u, cudaGraphCondAssignDefault)) != cudaSuccess) return e;
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        if ((e = cudaGraphAddNode(&node, g, deps, nd, &p)) != cudaSuccess) return e;
        cudaGraph_t bg = p.conditional.phGraph_out[0];
        if ((e = cudaStreamBeginCaptureToGraph(aux, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal)) !=
            cudaSuccess)
            return e;
        st = aux;
        body(h, 1);
        st = c.stream;
        if ((e = cudaStreamEndCapture(aux, &bg)) != cudaSuccess) return e;
        if ((e = cudaStreamUpdateCaptureDependencies(c.stream, &node, 1, cudaStreamSetCaptureDependencies)) !=
            cudaSuccess)
            return e;
    } else {
        for (int it = 0; it < max_iter; ++it) body(0, 0);
    }
    solveFinalKernel<<<ngrid, kThreads, 0, c.stream>>>(a);
    ++launches;
    noteLaunches(launches);
    return cudaGetLastError();
}

}  // namespace mpm
