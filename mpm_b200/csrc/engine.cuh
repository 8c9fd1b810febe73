// engine.cuh -- device-side data layout of the B200 MPM step.
//
// HBM layout (one scene):
//   particles : two ping-pong SoA buffers.  Buffer k holds NFIELDS float
//               planes of `cap` floats (x[3] v[3] Fe[9] Fp[9] B[9] tau[6]
//               mass vol0), plus pid (original index, u32) and mat (u16).
//               After every step the live buffer is sorted by cell key.
//   grid      : dense float4 v* (xyz, w = node mass) and, for PIC-FLIP,
//               float4 v; node index x + X*(y + Y*z).
//   keys      : per-particle u32 key = (global block << 6) | cell-in-block,
//               blocks are 4^3 cells of stencil bases, shifted by one block
//               so that bases down to -3 stay non-negative.
// Batch-wide scratch: radix-sort ping-pong keys/values, the active-block
// list, the dense block->slot map and the per-block P2G tiles.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mpm {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSortTileKeys = kThreads * 8;  // keys per radix-sort tile (8 per thread)
// Work items: a block's sorted particles are split into
// ceil(count / kBlockChunk) P2G items of nearly equal size (each with its own
// P2G tile, merged in item order), so that one crowded block cannot serialize
// a step.  The split fixes the order of P2G's sums, so it is a constant.
// (Splits of 2048 and 1024 particles were no faster on the dense two-ball
// scene -- P2G 0.150 and 0.144 ms against 0.145 ms -- and slowed the grid
// pass, which sums more tiles per node.)
constexpr uint32_t kBlockChunk = 4096;
// G2P has no sums across particles, so its work items can be smaller without
// changing any result: a block is split into ceil(count / chunk) G2P items,
// which balances the persistent CTAs better than P2G's items.  The chunk is an
// engine setting (autotuned) in [kMinG2PChunk, kMaxG2PChunk].
constexpr uint32_t kMinG2PChunk = 256;
constexpr uint32_t kMaxG2PChunk = 4096;
constexpr uint32_t kDefaultG2PChunk = 1024;
// Counter words: [0] work items, [1] outside items, [2] nodes with mass,
// [8 + 8k .. 13 + 8k] work-item schedulers of combination k (k < 6),
// [kG2PCountWord + k] G2P items of combination k.
constexpr int kMaxCombos = 6;
constexpr int kG2PCountWord = 56;
// [kP2GListWord + 2k + c]: P2G items of combination k in its list c (0: items
// of at most the warp threshold's particles, taken by whole warps; 1: the
// others, taken by whole CTAs); counter words in all: kCounterWords.
constexpr int kP2GListWord = 64;
// [kP2GSmallWord + k]: P2G items of combination k of at most kWarpAutoMax
// particles (read back to decide the warp threshold when it is not set).
constexpr int kP2GSmallWord = kP2GListWord + 2 * kMaxCombos;
// The CTA list (c = 1) of combination k holds its items of at least
// kBigItem particles from the front (counters[kP2GListWord + 2k + 1] of
// them) and the others from the back (counters[kP2GBackWord + k]), so that
// the CTAs take the long items first and the short ones fill the tail.
constexpr int kP2GBackWord = kP2GSmallWord + kMaxCombos;
constexpr uint32_t kBigItem = 1024;
constexpr uint32_t kWarpAutoMax = 256;
constexpr uint32_t kWarpAutoMinItems = 1024;
// Who takes the small P2G items (list 0) in a step: p2gKernel after its own
// list (no warp kernel launched), p2gWarpKernel, or -- decided on the device
// from the list's length, the same way by both kernels -- p2gWarpKernel when
// the list holds at least kWarpAutoMinItems items, else p2gKernel.
enum P2GWarp : int { P2G_WARP_NONE = 0, P2G_WARP_ALWAYS = 1, P2G_WARP_AUTO = 2 };
__host__ __device__ inline bool p2gWarpTakesSmall(int mode, uint32_t n_small) {
    return mode == P2G_WARP_ALWAYS || (mode == P2G_WARP_AUTO && n_small >= kWarpAutoMinItems);
}
constexpr int kCounterWords = 128;
static_assert(kP2GBackWord + kMaxCombos <= kCounterWords, "counter words");

enum Field : int {
    F_X = 0,
    F_V = 3,
    F_FE = 6,
    F_FP = 15,
    F_B = 24,
    F_TAU = 33,  // symmetric V0 * stress: xx yy zz xy xz yz
    F_MASS = 39,
    F_VOL = 40,
    NFIELDS = 41
};

// Device error flags (bit mask).
enum : uint32_t {
    ERR_NONFINITE = 1u,      // a particle position/velocity became NaN/Inf
    ERR_TILE_OVERFLOW = 2u,  // more active blocks than tile slots (never expected)
    ERR_INDEX = 4u,          // a permutation or stencil index failed its range check (never expected)
    ERR_WAIT_TIMEOUT = 64u,  // a bounded wait for a TMA tile gave up (never expected)
};

// Bytes of one TMA tensor map (CUtensorMap) and the device-side table of
// them: per scene, v* then v (PIC-FLIP; APIC repeats v*).
constexpr int kTensorMapBytes = 128;

struct ParticleBuf {
    float* f;        // NFIELDS * cap
    uint32_t* pid;   // cap
    uint16_t* mat;   // cap
};

// 16-byte aligned (sizeof 32) so that G2P can bulk-copy a scene's first
// material into shared memory.
struct alignas(16) MaterialDev {
    float mu0, lambda0, xi, theta_c, theta_s;
    int model;
};

// Per-scene CFL state in device memory: the running max of |v|^2 as float
// bits (non-negative floats order like their bit patterns), the dt of the
// last step and the simulated time it advanced.
struct CflState {
    uint32_t vmax2_bits;
    float last_dt;
    double time;
};

// Semi-implicit solve of one scene (see implicit.cu).  vec holds seven
// dense node vectors of float4 (x, r, z, p, Ap, Az, h; .w unused); list the
// nodes with mass; part the per-block FP64 partial sums of the dot
// products, [quantity][slot][block].
struct SolveStatus {
    int done_at;     // first iteration whose test found convergence (INT_MAX while running)
    int iters;
    float residual;  // |r| / |M v*| at the end
    int nactive;     // nodes in list
};
struct SolveDev {
    float* m;
    float4* vec;
    int* list;
    double* part;
    SolveStatus* status;
};

// 16-byte aligned (sizeof a multiple of 16) so that the block kernels can
// bulk-copy a scene's entry into shared memory.
struct alignas(16) SceneDev {
    float origin[3];
    float h, inv_h, range;
    float target[3];
    int res[3];
    int nb[3];             // blocks per axis
    uint32_t block_base;   // global id of this scene's first block
    uint32_t nblocks;      // nb.x*nb.y*nb.z; block_base + nblocks is the scene's "outside" block
    uint32_t key_offset;   // first global particle slot of this scene
    uint32_t n;            // particles
    uint32_t cap;          // plane stride of the particle buffers
    float dt, gravity, friction, blend, dinv;
    int transfer, interp, S, boundary, sticky, pcoll, nmat;
    int combo;             // index of the scene's (stencil, transfer) combination in the batch
    int init_pass;         // 1: the mass pass of initialize() covers this scene
    ParticleBuf buf[2];
    float4* vstar;         // dense res^3
    float4* vold;          // dense res^3 (PIC-FLIP)
    const MaterialDev* mats;
    float* dbg;            // split-mode dense grid: mass, vel[3], force[3], vstar[3] planes
    // Level-set collision object (the reference's LevelSetCollisionObject3D,
    // include/collision_object3d.h:9-12): signed distance sampled on the grid
    // nodes (index x + X(y + Y z), negative inside), or null.
    const float* phi;
    float phi_friction;
    float phi_vel[3];      // velocity of the collider's surface
    // CFL time step: cfl > 0 makes each step's dt = min(dt_max, cfl h / max|v_p|),
    // written into dt by cflFinalizeKernel before the step's kernels run.
    float cfl, dt_max;
    CflState* cfl_state;
    // semi-implicit update: beta > 0 makes the step solve
    // (M + beta dt^2 H) v = M v* after the grid collision
    float beta, solve_tol;
    int solve_max_iter;
    SolveDev solve;
};

struct BlockItem {
    uint32_t block;   // global block id
    uint32_t start;   // first sorted particle (global)
    uint32_t count;
    uint32_t scene;
};

// Per-step kernel arguments.
struct StepArgs {
    const SceneDev* scenes;
    int nscenes;
    int parity;                  // live particle buffer index
    const uint32_t* sorted_keys; // N
    const uint32_t* perm;        // N: sorted position -> global old slot
    const BlockItem* active;
    const BlockItem* g2p_items;  // G2P's finer work items: combination k's (any order) at
                                 // g2p_items + k * g2p_cap, counters[kG2PCountWord + k] of them
    uint32_t g2p_cap;
    int combo;                   // the combination a G2P launch serves
    const uint32_t* counters;    // [0] active blocks, [1] outside blocks
    const BlockItem* outside;
    const int32_t* block_slot;   // dense: block -> slot or -1
    float* tiles;                // [slot][F][TN]
    uint32_t tile_stride;        // floats per slot
    uint32_t* next_keys;         // N
    uint32_t* block_count;       // dense per block
    uint32_t* err;               // error flags
    uint32_t* stats;             // [2]: nodes with mass written by the grid pass
    uint32_t* sched;             // work-item schedulers: [0..1] P2G, [2..3] P2G by warps, [4..5] G2P
                                 // (zero between launches)
    const uint32_t* p2g_lists;   // P2G item slots of combination `combo`'s lists (see kP2GListWord):
                                 // list c at p2g_lists + (2 combo + c) p2g_list_cap; null: P2G
                                 // takes every item of the active list
    uint32_t p2g_list_cap;
    int p2g_warp;                // who takes list 0 (the small items): P2G_WARP_NONE, _ALWAYS or _AUTO
    const unsigned char* tmaps;  // kTensorMapBytes x 2 per scene (64-byte aligned): TMA maps of v*, v
    unsigned long long* spans;   // this combination's kernel time spans (see KernelSpan), or null
};

// Kernel time spans measured on the device inside the (graph-replayed) step:
// per (family, combination) four words -- [0] the earliest CTA start of the
// running launch (all ones between launches), [1] the sum of the launches'
// spans in ns, [2] their count, [3] CTAs finished in the running launch.  The
// last CTA to finish closes the span (%globaltimer, nanoseconds).
enum KernelSpan : int { SPAN_P2G = 0, SPAN_GRID = 1, SPAN_G2P = 2, SPAN_FAMILIES = 3 };
constexpr int kSpanWords = 4 * SPAN_FAMILIES;  // per combination
__device__ __forceinline__ unsigned long long globalTimerNs() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
__device__ __forceinline__ void spanBegin(unsigned long long* spans, int family) {
    if (spans && threadIdx.x == 0) atomicMin(&spans[4 * family], globalTimerNs());
}
// `counted`: the launch counts as one more of the family's launches (a
// second launch of a family in the same step adds its time only).
__device__ __forceinline__ void spanEnd(unsigned long long* spans, int family, bool counted = true) {
    if (spans && threadIdx.x == 0) {
        unsigned long long* sp = spans + 4 * family;
        __threadfence();
        if (atomicAdd(&sp[3], 1ull) == (unsigned long long)gridDim.x - 1) {
            const unsigned long long t1 = globalTimerNs();
            const unsigned long long t0 = atomicExch(&sp[0], ~0ull);
            sp[1] += t1 - t0;
            if (counted) sp[2] += 1;
            sp[3] = 0;
        }
    }
}

// Dynamic work-item scheduler of the persistent block kernels: sched[0]
// hands out item indices, sched[1] counts the CTAs that have run out; the
// last of those clears both, so every launch starts from zero without a
// memset.  Call from all threads of the CTA; returns the CTA's next item.
__device__ __forceinline__ uint32_t nextWorkItem(uint32_t* sched, uint32_t total, uint32_t* slot) {
    __syncthreads();  // the previous item's shared memory is no longer read
    if (threadIdx.x == 0) {
        const uint32_t w = atomicAdd(&sched[0], 1u);
        if (w >= total && atomicAdd(&sched[1], 1u) == gridDim.x - 1) {
            sched[0] = 0u;
            sched[1] = 0u;
        }
        *slot = w;
    }
    __syncthreads();
    return *slot;
}

// P2G/grid-pass variants.
enum P2GMode : int {
    MODE_APIC_FUSED = 0,  // fields: m, p + dt f        (F = 4)
    MODE_FLIP = 1,        // fields: m, p, f            (F = 7)
    MODE_SPLIT = 2,       // fields: m, p, f (any transfer, split API, F = 7)
    MODE_MASS = 3         // fields: m                  (F = 1)
};

__host__ __device__ constexpr int modeFields(int mode) {
    return mode == MODE_APIC_FUSED ? 4 : (mode == MODE_MASS ? 1 : 7);
}
__host__ __device__ constexpr int tileNodes(int S) { return (S + 3) * (S + 3) * (S + 3); }

}  // namespace mpm
