// engine_host.hpp -- host-side launch interface between the engine and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/mpm_b200.h"
#include "engine.cuh"

namespace mpm {

struct LaunchCtx {
    const SceneDev* scenes;   // device scene table
    int nscenes;
    cudaStream_t stream;
    unsigned particle_blocks;   // grid.x of per-particle kernels (grid.y = scene)
    unsigned node_blocks;       // grid.x of dense per-node kernels
    unsigned persistent_blocks; // grid of the persistent block kernels
    int num_sms;
    int p2g_stage;              // particles staged per warp pass in P2G (16 or 32)
};

struct BlockBuffers {
    uint32_t* block_count;            // total_blocks
    uint32_t* scene_block_base;       // nscenes + 1
    BlockItem* active;                // max_active
    BlockItem* outside;               // nscenes
    BlockItem* g2p_items;             // G2P work items, g2p_cap per combination
    uint32_t g2p_cap;
    uint32_t* counters;               // see kG2PCountWord, kP2GListWord
    int32_t* block_slot;              // total_blocks
    uint32_t* p2g_lists;              // P2G item slots, 2 lists of p2g_list_cap per combination
    uint32_t p2g_list_cap;
};

// Host-side count of kernel launches issued by the library (kernels.cu).
void noteLaunches(uint64_t n);
uint64_t kernelLaunches();

// sort.cu
// Up to four word ranges zeroed by one kernel launch (launchClear): the
// step's scratch clears are kernels rather than memset nodes, which a
// device-to-host copy running beside the step (an asynchronous download on
// another stream) held back by 8-20 us each.
struct ClearRanges {
    uint32_t* p[4] = {};
    size_t n[4] = {};
};
void launchClear(const ClearRanges& r, cudaStream_t st);
size_t scanScratchElems(size_t n);
template <class T>
cudaError_t exclusiveScan(const T* in, T* out, size_t n, T* partials, T* total, cudaStream_t st);
size_t radixTiles(size_t n);
size_t onesweepScratchWords(size_t n, int bits);
cudaError_t radixSortOnesweep(uint32_t* keys_a, uint32_t* vals_a, uint32_t* keys_b, uint32_t* vals_b, size_t n,
                              int bits, uint32_t* scratch, uint32_t* err, bool* result_in_b, cudaStream_t st,
                              const uint32_t* n_dev = nullptr);
// Incremental sort (sort.cu): the stable sort of `keys` (n, live order) given
// that `prev` (the previous step's sorted keys, aligned with the same live
// order) is ascending.  Output equals radixSortOnesweep's (keys, perm).
size_t incrementalSortScratchWords(size_t n, int bits);
cudaError_t incrementalSort(const uint32_t* keys, const uint32_t* prev, size_t n, int bits, uint32_t* out_keys,
                            uint32_t* out_perm, uint32_t* scratch, uint32_t* err, cudaStream_t st);
cudaError_t radixSortPairsInto(const uint32_t* in_keys, uint32_t* out_keys, uint32_t* out_vals, uint32_t* tmp_keys,
                               uint32_t* tmp_vals, size_t n, int bits, uint32_t* hist, uint32_t* scan_partials,
                               cudaStream_t st);

// kernels.cu
void launchKeys(const LaunchCtx& c, int parity, uint32_t* keys, uint32_t* block_count, uint32_t* err);
size_t compactScratchWords64(uint32_t total_blocks);
// How the compaction splits each (stencil, transfer) combination's work:
// particles per G2P work item, and the largest P2G item taken by a single
// warp (0: none).
struct ComboSplit {
    uint32_t g2p_chunk[kMaxCombos];
    uint32_t p2g_warp_max[kMaxCombos];
};
void launchCompactOnesweep(const LaunchCtx& c, const BlockBuffers& bb, uint32_t total_blocks,
                           unsigned long long* scratch, uint32_t chunk, const ComboSplit& split, uint32_t* err);
void launchStress(const LaunchCtx& c, int parity);
void launchP2G(const LaunchCtx& c, const StepArgs& a, int S, int mode, int want_transfer);
// P2G of the combination a.combo's warp list (a.p2g_lists set): one warp per
// item, tiles bitwise those of launchP2G.
void launchP2GWarp(const LaunchCtx& c, const StepArgs& a, int S, int mode);
void launchGrid(const LaunchCtx& c, const StepArgs& a, int S, int mode, int want_transfer);
void launchG2P(const LaunchCtx& c, const StepArgs& a, int S, bool apic, bool fused, int combo);
void launchDenseGravity(const LaunchCtx& c);
void launchDenseUpdate(const LaunchCtx& c, float dt);
void launchDenseCollision(const LaunchCtx& c, float dt);
void launchDensePack(const LaunchCtx& c);
void launchParticlesCollision(const LaunchCtx& c, int parity, float dt);
void launchAdvect(const LaunchCtx& c, int parity, float dt);
void launchVolume(const LaunchCtx& c, int parity, int S);
// A new scene's particle planes from its staged arrays, slot i from the
// caller's particle perm[i] (perm null: i); mat_in null: no material ids.
void launchInitState(cudaStream_t st, int num_sms, float* f, uint32_t* pid, uint16_t* mat, size_t cap,
                     const float* staged, size_t n, bool has_volume, const uint32_t* perm, const uint16_t* mat_in);
// Cell keys (sc's block numbering) of n staged interleaved positions.
void launchStagedKeys(cudaStream_t st, int num_sms, const SceneDev& sc, const float* xyz, uint32_t n, uint32_t* keys,
                      uint32_t* err);
void launchDensity(const LaunchCtx& c, const float4* vstar, size_t nodes, float inv_cell_vol, float* out);
// Semi-implicit solve (implicit.cu) of the scenes with beta > 0.  Global
// buffers over the sorted particles of the batch and its cell keys.
struct SolveBuffers {
    const uint32_t* sorted_keys;  // ntot
    const uint32_t* perm;         // ntot
    uint2* cell_range;            // nkeys: first and end sorted position of each cell key
    size_t nkeys;
    uint2* block_range;           // nblocks: the same per 4^3 block of cells (key >> 6)
    size_t nblocks;
    float4* pofs;                 // ntot: stencil offsets (x - (o + h base)) / h (sorted order)
    float* prep;                  // kSolvePrepPlanes x ntot
    float4* T;                    // 3 x ntot: V0 dP Fe^T rows
    uint32_t ntot;
    int* iter;                    // device iteration counter
};
constexpr int kSolvePrepPlanes = 44;
constexpr int kSolveVectors = 7;
constexpr int kSolveBlocks = 512;  // node-kernel blocks per scene = partial sums per dot product
inline size_t solvePartialDoubles(int max_iter) { return (size_t)4 * (size_t)(max_iter + 2) * kSolveBlocks; }
// split: v* from and to the split-mode dense planes (no collision after);
// else from and to the fused step's v* grid, with the grid collision after.
// aux: an idle stream on which, inside a stream capture, the iteration body
// is captured as the body of a conditional while node.
cudaError_t launchSolve(const LaunchCtx& c, const SolveBuffers& b, int parity, const int* stencils, int nstencils,
                        int max_iter, bool split, cudaStream_t aux);

// CFL time step of the scenes with cfl > 0: max |v|^2 over their live
// particles, then dt = min(dt_max, cfl h / max|v|) into the scene table.
// A non-finite particle speed sets ERR_NONFINITE in err.
void launchCfl(const LaunchCtx& c, int parity, size_t max_n, uint32_t* err);
void launchGatherField(const LaunchCtx& c, int scene, int parity, int field, int comps, int mode, float* out);
void preloadTransferKernels();
void launchScatterField(const LaunchCtx& c, int scene, int parity, int field, int comps, const float* in);
size_t p2gSmemBytes(int S, int mode);
// Writes the kTensorMapBytes TMA tensor map of a dense float4 grid (res[3]
// nodes) with tile box T^3 to map (host memory); returns null or a message.
const char* encodeGridTensorMap(void* map, const void* grid, const int* res, int T);

}  // namespace mpm
