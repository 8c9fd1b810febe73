// engine.cu -- host engine: scene batches, device memory, step orchestration,
// and the C ABI declared in include/mpm_b200.h.
//
// A solver handle (mpm_solver) is an Engine holding one scene; a batch
// (mpm_batch, include/mpm_b200_batch.h) holds many.  Every step of a batch is
// one sequence of launches on the engine's stream:
//   [keys] -> radix sort -> block compaction -> [stress] -> P2G -> grid -> G2P
// where the bracketed kernels only run after uploads or split-API calls
// (in steady state G2P produces next step's keys and stress).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <sys/stat.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <deque>
#include <map>
#include <set>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"
#include "../../include/mpm_b200_batch.h"
#include "engine_host.hpp"

namespace mpm {

static thread_local std::string g_last_error;

static mpm_status fail(mpm_status st, const std::string& msg) {
    g_last_error = msg;
    return st;
}

// Error recording for entry points defined in other translation units.
mpm_status recordError(mpm_status st, const char* msg) { return fail(st, msg ? msg : ""); }
mpm_status writeDensityVdb(const float* density, const int32_t* res, const char* path);  // vdb.cpp

#define CUDA_TRY(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) {                                                                       \
            return fail(e_ == cudaErrorMemoryAllocation ? MPM_ERR_OOM : MPM_ERR_CUDA,                  \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
        }                                                                                              \
    } while (0)

#define MPM_TRY(call)                  \
    do {                               \
        mpm_status s_ = (call);        \
        if (s_ != MPM_OK) return s_;   \
    } while (0)

enum KernelFamily { KF_KEYS = 0, KF_SORT, KF_COMPACT, KF_STRESS, KF_P2G, KF_GRID, KF_G2P, KF_COUNT };

// Scenes of at least this many particles are uploaded in cell-sorted order.
constexpr size_t kSortedUploadMin = (size_t)1 << 16;

static int stencilSize(int interp) {
    return interp == MPM_INTERP_LINEAR ? 2 : (interp == MPM_INTERP_QUADRATIC_BSPLINE ? 3 : 4);
}
static float stencilRange(int interp) {
    return interp == MPM_INTERP_LINEAR ? 1.0f : (interp == MPM_INTERP_QUADRATIC_BSPLINE ? 1.5f : 2.0f);
}

// Per-device stream-ordered memory pool for scene state.  Freed blocks stay
// in the pool (release threshold: unlimited), so scenes that come and go in
// a batch or a server reuse device memory without cudaMalloc/cudaFree and
// their device-wide synchronisation.  mpm_release_cached_memory() returns
// the unused part to the driver.
static cudaMemPool_t scenePool(int device, mpm_status* st) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    std::lock_guard<std::mutex> lock(mu);
    if (device < 0 || device >= 64) {
        *st = fail(MPM_ERR_INVALID_ARG, "device index out of range");
        return nullptr;
    }
    if (!pools[device]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
        if (e != cudaSuccess) {
            cudaGetLastError();
            *st = fail(MPM_ERR_CUDA, std::string("memory pool: ") + cudaGetErrorString(e));
            return nullptr;
        }
        pools[device] = pool;
    }
    *st = MPM_OK;
    return pools[device];
}

// Streams of destroyed engines, kept per device for the next engines (a
// solver that is created per request, a benchmark's repeated constructions):
// creating a stream costs about 0.1 ms, taking an idle one nothing.  A
// stream is given back after its engine's last synchronize; what it still
// holds (stream-ordered frees to the pool) runs before the next owner's work.
static std::mutex g_stream_mu;
static std::vector<std::pair<int, cudaStream_t>> g_idle_streams;
constexpr size_t kMaxIdleStreams = 64;

static cudaError_t takeStream(int device, cudaStream_t* s) {
    {
        std::lock_guard<std::mutex> lock(g_stream_mu);
        for (size_t i = g_idle_streams.size(); i-- > 0;)
            if (g_idle_streams[i].first == device) {
                *s = g_idle_streams[i].second;
                g_idle_streams.erase(g_idle_streams.begin() + (long)i);
                return cudaSuccess;
            }
    }
    return cudaStreamCreateWithFlags(s, cudaStreamNonBlocking);
}

static void giveStream(int device, cudaStream_t s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(g_stream_mu);
        if (g_idle_streams.size() < kMaxIdleStreams) {
            g_idle_streams.push_back({device, s});
            return;
        }
    }
    cudaStreamDestroy(s);
}

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    cudaStream_t pool_stream = nullptr;  // set: memory of the scene pool, freed in this stream's order
    ~DevMem() { release(); }
    void release() {
        if (p) {
            if (pool_stream) cudaFreeAsync(p, pool_stream);
            else cudaFree(p);
        }
        p = nullptr;
        bytes = 0;
        pool_stream = nullptr;
    }
    // Grow to at least b bytes, by at least half the current size, so that a
    // batch whose scenes come and go rarely reallocates.
    mpm_status grow(size_t b, const char* what) {
        if (p && bytes >= b) return MPM_OK;
        return alloc(std::max(b, bytes + bytes / 2), what);
    }
    mpm_status alloc(size_t b, const char* what) {
        if (p && bytes >= b) return MPM_OK;
        release();
        if (b == 0) b = 16;
        cudaError_t e = cudaMalloc(&p, b);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(MPM_ERR_OOM, std::string("cudaMalloc failed for ") + what + " (" + std::to_string(b) + " bytes)");
        }
        bytes = b;
        return MPM_OK;
    }
    // From the scene pool, in the order of `stream` (the engine's stream; the
    // memory is usable there at once and elsewhere after an event on it).
    mpm_status allocPooled(size_t b, const char* what, cudaMemPool_t pool, cudaStream_t stream) {
        if (p && bytes >= b) return MPM_OK;
        release();
        if (b == 0) b = 16;
        cudaError_t e = cudaMallocFromPoolAsync(&p, b, pool, stream);
        if (e != cudaSuccess) {
            p = nullptr;
            cudaGetLastError();
            return fail(MPM_ERR_OOM, std::string("pool allocation failed for ") + what + " (" + std::to_string(b) +
                                         " bytes)");
        }
        bytes = b;
        pool_stream = stream;
        return MPM_OK;
    }
    template <class T>
    T* as() const {
        return (T*)p;
    }
};

struct SceneHost {
    int id = -1;
    mpm_scene_desc desc{};
    size_t n = 0;
    int S = 4;
    int nb[3] = {0, 0, 0};
    uint32_t nblocks = 0;
    DevMem buf_f[2], buf_pid[2], buf_mat[2];
    DevMem vstar, vold, dbg, mats;
    int nmat = 1;
    bool need_init = true;
    bool stress_stale = true;  // cached tau must be recomputed from Fe/Fp
    // asynchronous downloads: two staging buffers, each with the event of its
    // gather (ready) and of its copy to the host (done)
    DevMem stage[2];
    cudaEvent_t stage_ready[2] = {}, stage_done[2] = {};
    bool stage_pending[2] = {};
    int stage_next = 0;
    std::vector<mpm_material> mats_in;  // as given (kept for checkpoints)
    DevMem phi;                         // level-set collision object (nodes floats), if set
    bool has_phi = false;
    float phi_friction = 0.f, phi_vel[3] = {0.f, 0.f, 0.f};
    // simulated time: steps at the fixed dt are counted here, CFL steps on the
    // device (CflState); last_cfl tells which holds the last step's dt
    float cfl = 0.f;
    DevMem cfl_state;
    double time_fixed = 0.0;
    float last_dt = 0.f;
    bool last_cfl = false;
    // semi-implicit update (beta > 0) and its solver buffers (implicit.cu)
    float beta = 0.f, solve_tol = 1e-5f;
    int solve_max_iter = 50;
    DevMem solve_m, solve_vec, solve_list, solve_part, solve_status;
    size_t nodes() const { return (size_t)desc.resolution[0] * desc.resolution[1] * desc.resolution[2]; }
    ~SceneHost() {
        for (int k = 0; k < 2; ++k) {
            if (stage_done[k]) {
                cudaEventSynchronize(stage_done[k]);  // no copy may still read the staging buffer
                cudaEventDestroy(stage_done[k]);
            }
            if (stage_ready[k]) cudaEventDestroy(stage_ready[k]);
        }
    }
};

// ---------------------------------------------------------------------------
// Page-locked host words for asynchronous read-backs of single device words
// (the P2G staging decision).  One page-locked block for the process, handed
// out word by word: cudaHostAlloc per engine costs milliseconds (it pins
// pages), which a solver's construction and first step would pay.
// ---------------------------------------------------------------------------
struct PinnedWords {
    std::mutex mu;
    uint32_t* base = nullptr;
    std::vector<int> free_slots;
    static constexpr int kSlots = 4096;
    static constexpr int kLine = 8;  // words per slot
    uint32_t* take() {  // kLine contiguous words
        std::lock_guard<std::mutex> lock(mu);
        if (!base) {
            if (cudaHostAlloc((void**)&base, sizeof(uint32_t) * kSlots * kLine, cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                base = nullptr;
                return nullptr;
            }
            for (int i = kSlots - 1; i >= 0; --i) free_slots.push_back(i);
        }
        if (free_slots.empty()) return nullptr;
        const int i = free_slots.back();
        free_slots.pop_back();
        return base + (size_t)i * kLine;
    }
    void give(uint32_t* p) {
        std::lock_guard<std::mutex> lock(mu);
        if (p && base) free_slots.push_back((int)((p - base) / kLine));
    }
};
static PinnedWords g_pinned_words;

// ---------------------------------------------------------------------------
// Tuning cache of the autotuner: launch settings per (device, stencil size,
// transfer, particles-per-cell bucket), kept for the process and in a text
// file ("<device> <S> <transfer> <bucket> <g2p_chunk> <p2g_stage>" per line;
// the last line of a key wins).
// ---------------------------------------------------------------------------
struct TuneCache {
    std::mutex mu;
    std::map<std::string, mpm_tuning> entries;
    bool loaded = false;

    static std::string path() {
        if (const char* e = getenv("MPM_TUNE_CACHE")) return e;
        std::string dir;
        if (const char* x = getenv("XDG_CACHE_HOME")) dir = x;
        else if (const char* h = getenv("HOME")) dir = std::string(h) + "/.cache";
        else return "";
        return dir + "/mpm_b200/tuning.txt";
    }
    static std::string key(const std::string& dev, int S, int transfer, int bucket) {
        return dev + " " + std::to_string(S) + " " + std::to_string(transfer) + " " + std::to_string(bucket);
    }
    void load() {
        if (loaded) return;
        loaded = true;
        const std::string p = path();
        if (p.empty()) return;
        FILE* f = fopen(p.c_str(), "r");
        if (!f) return;
        // one entry per line; lines of an older format (fewer values) are
        // skipped, so their keys are tuned again
        char line[512], dev[256];
        int S, tr, bucket, chunk, stage, warp;
        while (fgets(line, sizeof(line), f))
            if (sscanf(line, "%255s %d %d %d %d %d %d", dev, &S, &tr, &bucket, &chunk, &stage, &warp) == 7 &&
                chunk >= (int)kMinG2PChunk && chunk <= (int)kMaxG2PChunk && (stage == 16 || stage == 24 || stage == 32) &&
                warp >= -1 && warp <= MPM_P2G_WARP_MAX_MAX)
                entries[key(dev, S, tr, bucket)] = mpm_tuning{chunk, stage, warp};
        fclose(f);
    }
    void store(const std::string& k, const mpm_tuning& t, bool disk) {
        entries[k] = t;
        if (!disk) return;
        const std::string p = path();
        if (p.empty()) return;
        // create the directories of the path (best effort)
        for (size_t i = 1; i < p.size(); ++i)
            if (p[i] == '/') mkdir(p.substr(0, i).c_str(), 0755);
        if (FILE* f = fopen(p.c_str(), "a")) {
            fprintf(f, "%s %d %d %d\n", k.c_str(), t.g2p_chunk, t.p2g_stage, t.p2g_warp_max);
            fclose(f);
        }
    }
};
static TuneCache g_tune_cache;

class Engine {
public:
    struct GraphSlot {
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
    };
    Engine() {}
    ~Engine() {
        if (stream_) cudaStreamSynchronize(stream_);
        if (copy_stream_) cudaStreamSynchronize(copy_stream_);
        scenes_.clear();  // their staging events before the copy stream
        giveStream(device_, copy_stream_);
        dropGraphs();
        for (int k = 0; k < KF_COUNT; ++k) {
            if (ev_[k][0]) cudaEventDestroy(ev_[k][0]);
            if (ev_[k][1]) cudaEventDestroy(ev_[k][1]);
            if (open_[k]) cudaEventDestroy(open_[k]);
        }
        for (auto& r : records_) {
            cudaEventDestroy(r.e0);
            cudaEventDestroy(r.e1);
        }
        for (auto e : event_pool_) cudaEventDestroy(e);
        for (int k = 0; k < kMaxSide; ++k) {
            if (side_[k]) {
                cudaStreamSynchronize(side_[k]);
                giveStream(device_, side_[k]);
            }
            if (join_[k]) cudaEventDestroy(join_[k]);
        }
        if (fork_) cudaEventDestroy(fork_);
        if (compact_stream_) {
            cudaStreamSynchronize(compact_stream_);
            giveStream(device_, compact_stream_);
        }
        if (compact_fork_) cudaEventDestroy(compact_fork_);
        if (compact_join_) cudaEventDestroy(compact_join_);
        releaseScratch();
        for (auto& p : step_events_) {
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        for (auto e : free_events_) cudaEventDestroy(e);
        for (auto& e4 : tune_ev_)
            for (auto e : e4)
                if (e) cudaEventDestroy(e);
        if (host_word_) g_pinned_words.give(host_word_);
        if (stage_event_) cudaEventDestroy(stage_event_);
        giveStream(device_, stream_);
    }

    // Device memory of the engine (batch scratch, scene buffers) comes from
    // the per-device stream-ordered pool in the order of the engine's stream:
    // engines that are created and destroyed (solvers of a server, the
    // benchmark's repeated constructions) reuse memory without cudaMalloc or
    // the implicit device synchronization of cudaFree.
    mpm_status alloc(DevMem& m, size_t b, const char* what) { return m.allocPooled(b, what, pool_, stream_); }
    mpm_status grow(DevMem& m, size_t b, const char* what) {
        if (m.p && m.bytes >= b) return MPM_OK;
        return m.allocPooled(std::max(b, m.bytes + m.bytes / 2), what, pool_, stream_);
    }
    // Returns the engine's own buffers to the pool in the stream's order
    // (called before the stream is destroyed).
    void releaseScratch() {
        DevMem* all[] = {&cell_range_, &block_range_, &solve_pofs_, &solve_prep_, &solve_T_, &solve_iter_,
                         &keys_[0], &keys_[1], &vals_[0], &vals_[1], &sort_scratch_, &inc_scratch_,
                         &compact_scratch_, &block_count_, &sbb_, &active_, &outside_, &counters_, &block_slot_,
                         &tiles_, &scenes_dev_, &err_, &tmp_, &g2p_items_, &tmaps_, &spans_, &p2g_lists_};
        for (DevMem* m : all) m->release();
    }

    mpm_status init() {
        CUDA_TRY(cudaGetDevice(&device_));
        {
            mpm_status pst;
            pool_ = scenePool(device_, &pst);
            if (!pool_) return pst;
        }
        CUDA_TRY(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, device_));
        {   // the host-transfer kernels, once per device (see preloadTransferKernels)
            static std::mutex mu;
            static std::set<int> done;
            std::lock_guard<std::mutex> lock(mu);
            if (done.insert(device_).second) preloadTransferKernels();
        }
        CUDA_TRY(takeStream(device_, &stream_));
        CUDA_TRY(takeStream(device_, &compact_stream_));
        CUDA_TRY(cudaEventCreateWithFlags(&compact_fork_, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&compact_join_, cudaEventDisableTiming));
        MPM_TRY(alloc(err_, sizeof(uint32_t), "error flags"));
        CUDA_TRY(cudaMemsetAsync(err_.p, 0, sizeof(uint32_t), stream_));
        for (int k = 0; k < KF_COUNT; ++k) {
            CUDA_TRY(cudaEventCreate(&ev_[k][0]));
            CUDA_TRY(cudaEventCreate(&ev_[k][1]));
        }
        return MPM_OK;
    }

    static mpm_status validate(const mpm_scene_desc& d, const mpm_particles_in& p) {
        for (int a = 0; a < 3; ++a)
            if (d.resolution[a] <= 0 || d.resolution[a] > (1 << 16))
                return fail(MPM_ERR_INVALID_ARG, "grid resolution must be in [1, 65536]");
        if (!(d.stride > 0.f) || !std::isfinite(d.stride)) return fail(MPM_ERR_INVALID_ARG, "stride must be > 0");
        if (!(d.dt > 0.f) || !std::isfinite(d.dt)) return fail(MPM_ERR_INVALID_ARG, "dt must be > 0");
        if (d.interpolation < MPM_INTERP_LINEAR || d.interpolation > MPM_INTERP_CUBIC_BSPLINE)
            return fail(MPM_ERR_INVALID_ARG, "unsupported interpolation type");
        if (d.transfer != MPM_TRANSFER_PIC_FLIP && d.transfer != MPM_TRANSFER_APIC)
            return fail(MPM_ERR_INVALID_ARG, "unsupported transfer");
        if (d.transfer == MPM_TRANSFER_APIC && d.interpolation == MPM_INTERP_LINEAR)
            return fail(MPM_ERR_INVALID_ARG,
                        "APIC with linear interpolation has a singular inertia tensor D (reference leaves it TODO)");
        if (d.boundary != MPM_BOUNDARY_REFERENCE && d.boundary != MPM_BOUNDARY_STICKY)
            return fail(MPM_ERR_INVALID_ARG, "unsupported boundary mode");
        if (d.boundary == MPM_BOUNDARY_STICKY && d.sticky_cells < 0)
            return fail(MPM_ERR_INVALID_ARG, "sticky_cells must be >= 0");
        if (d.volume_mode != MPM_VOLUME_GRID_ESTIMATE && d.volume_mode != MPM_VOLUME_PRESCRIBED)
            return fail(MPM_ERR_INVALID_ARG, "unsupported volume mode");
        if (p.n > 0 && (!p.position || !p.velocity || !p.mass))
            return fail(MPM_ERR_INVALID_ARG, "particle position, velocity and mass arrays are required");
        if (p.n > (size_t)0x7fffffff) return fail(MPM_ERR_INVALID_ARG, "too many particles");
        if (d.volume_mode == MPM_VOLUME_PRESCRIBED && p.n > 0 && !p.volume)
            return fail(MPM_ERR_INVALID_ARG, "prescribed volume mode needs a volume array");
        if (p.nmaterials < 1 || !p.materials) return fail(MPM_ERR_INVALID_ARG, "at least one material is required");
        if (p.nmaterials > 1 && p.n > 0 && !p.material)
            return fail(MPM_ERR_INVALID_ARG, "per-particle material ids are required with several materials");
        if (p.nmaterials > 65535) return fail(MPM_ERR_INVALID_ARG, "too many materials");
        for (int i = 0; i < p.nmaterials; ++i) {
            const mpm_material& m = p.materials[i];
            if (m.model != MPM_MODEL_FIXED_COROTATED && m.model != MPM_MODEL_NEO_HOOKEAN)
                return fail(MPM_ERR_INVALID_ARG, "unsupported constitutive model");
            if (!(m.poisson_ratio < 0.5f) || !(m.poisson_ratio > -1.0f))
                return fail(MPM_ERR_INVALID_ARG, "Poisson ratio must be in (-1, 0.5)");
        }
        if (p.material)
            for (size_t i = 0; i < p.n; ++i)
                if (p.material[i] >= p.nmaterials) return fail(MPM_ERR_INVALID_ARG, "material id out of range");
        return MPM_OK;
    }

    // A new scene's device buffers and material table (state not yet set).
    mpm_status newScene(const mpm_scene_desc& d, const mpm_material* materials, int nmaterials, size_t n,
                        std::unique_ptr<SceneHost>* out) {
        auto sc = std::make_unique<SceneHost>();
        sc->desc = d;
        sc->n = n;
        sc->S = stencilSize(d.interpolation);
        for (int a = 0; a < 3; ++a) sc->nb[a] = ((d.resolution[a] + 3) >> 2) + 1;
        sc->nblocks = (uint32_t)sc->nb[0] * sc->nb[1] * sc->nb[2];
        sc->mats_in.assign(materials, materials + nmaterials);
        const size_t cap = std::max<size_t>(n, 1);
        mpm_status pst;
        cudaMemPool_t pool = scenePool(device_, &pst);
        if (!pool) return pst;
        for (int b = 0; b < 2; ++b) {
            MPM_TRY(sc->buf_f[b].allocPooled(sizeof(float) * NFIELDS * cap, "particle state", pool, stream_));
            MPM_TRY(sc->buf_pid[b].allocPooled(sizeof(uint32_t) * cap, "particle ids", pool, stream_));
            MPM_TRY(sc->buf_mat[b].allocPooled(sizeof(uint16_t) * cap, "particle materials", pool, stream_));
            // With one material G2P does not copy the material ids between the
            // buffers, so both start as material 0 (pool memory is reused and
            // holds earlier contents); checkpoints save the plane as it is.
            CUDA_TRY(cudaMemsetAsync(sc->buf_mat[b].p, 0, sizeof(uint16_t) * cap, stream_));
        }
        const size_t nodes = sc->nodes();
        MPM_TRY(alloc(sc->cfl_state, sizeof(CflState), "CFL state"));
        CUDA_TRY(cudaMemsetAsync(sc->cfl_state.p, 0, sizeof(CflState), stream_));
        MPM_TRY(sc->vstar.allocPooled(sizeof(float4) * nodes, "grid v*", pool, stream_));
        CUDA_TRY(cudaMemsetAsync(sc->vstar.p, 0, sizeof(float4) * nodes, stream_));
        if (d.transfer == MPM_TRANSFER_PIC_FLIP) {
            MPM_TRY(sc->vold.allocPooled(sizeof(float4) * nodes, "grid v", pool, stream_));
            CUDA_TRY(cudaMemsetAsync(sc->vold.p, 0, sizeof(float4) * nodes, stream_));
        }
        // Materials: Lame parameters as in src/material_point3d.cu:25-26.
        std::vector<MaterialDev> mats(nmaterials);
        for (int i = 0; i < nmaterials; ++i) {
            const mpm_material& m = materials[i];
            double E = m.youngs_modulus, nu = m.poisson_ratio;
            mats[i].mu0 = (float)(E / (2.0 * (1.0 + nu)));
            mats[i].lambda0 = (float)((double)(m.youngs_modulus * m.poisson_ratio) / ((1.0 + nu) * (1.0 - 2.0 * nu)));
            mats[i].xi = m.hardening;
            mats[i].theta_c = m.critical_compression;
            mats[i].theta_s = m.critical_stretch;
            mats[i].model = m.model;
        }
        sc->nmat = nmaterials;
        MPM_TRY(sc->mats.allocPooled(sizeof(MaterialDev) * mats.size(), "materials", pool, stream_));
        // from pageable memory: the copy has taken the data when it returns,
        // so the host table may be freed without waiting for the stream
        CUDA_TRY(cudaMemcpyAsync(sc->mats.p, mats.data(), sizeof(MaterialDev) * mats.size(), cudaMemcpyHostToDevice,
                                 stream_));
        *out = std::move(sc);
        return MPM_OK;
    }

    static bool anyPinned(std::initializer_list<const void*> ptrs) {
        for (const void* p : ptrs) {
            if (!p) continue;
            cudaPointerAttributes a{};
            if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
                cudaGetLastError();
                return true;  // unknown: wait to be safe
            }
            if (a.type != cudaMemoryTypeUnregistered) return true;
        }
        return false;
    }

    int registerScene(std::unique_ptr<SceneHost> sc) {
        sc->id = next_id_++;
        const int id = sc->id;
        scenes_.push_back(std::move(sc));
        dirty_ = true;
        keys_valid_ = false;
        sorted_valid_ = false;
        return id;
    }

    mpm_status addScene(const mpm_scene_desc& d, const mpm_particles_in& p, int* out_id) {
        MPM_TRY(validate(d, p));
        std::unique_ptr<SceneHost> sc;
        MPM_TRY(newScene(d, p.materials, p.nmaterials, p.n, &sc));
        const size_t cap = std::max<size_t>(p.n, 1);
        // The caller's arrays are copied as they are (x, v interleaved; m; V0
        // if prescribed; material ids) into a staging buffer and a kernel
        // writes the SoA planes (Fe = Fp = I, B = 0).  A large scene is
        // written in cell-sorted order (pid keeps the caller's indices), the
        // order its first step's P2G, grid and G2P read it in: in the
        // caller's order (a random order, say) those gathers touch a new
        // sector per particle and the first step costs three steady ones.
        // The order of equal keys is the caller's, as in the step's stable
        // sort, so the scene's steps are the same to the bit.
        if (p.n > 0) {
            const bool has_vol = d.volume_mode == MPM_VOLUME_PRESCRIBED;
            const size_t n = p.n;
            const size_t mat_off = (sizeof(float) * (has_vol ? 8 : 7) * n + 15) / 16 * 16;
            MPM_TRY(grow(tmp_, mat_off + (p.material ? sizeof(uint16_t) * n : 0), "particle upload buffer"));
            float* staged = tmp_.as<float>();
            uint16_t* staged_mat = p.material ? (uint16_t*)((char*)tmp_.p + mat_off) : nullptr;
            const bool sorted = n >= kSortedUploadMin && n < ((size_t)1 << 30);
            // On an error return below, copies already queued still read the
            // caller's arrays: wait for them first.
            struct Drain {
                cudaStream_t a, b;
                bool on;
                ~Drain() {
                    if (on) {
                        cudaStreamSynchronize(a);
                        cudaStreamSynchronize(b);
                    }
                }
            } drain{stream_, compact_stream_, true};
            CUDA_TRY(cudaMemcpyAsync(staged, p.position, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, stream_));
            // With the sort, the other arrays follow the positions on the
            // compaction stream (idle here), so that the positions' keys and
            // sort run while they cross the bus.
            cudaStream_t rest = stream_;
            if (sorted) {
                CUDA_TRY(cudaEventRecord(compact_fork_, stream_));
                CUDA_TRY(cudaStreamWaitEvent(compact_stream_, compact_fork_, 0));
                rest = compact_stream_;
            }
            CUDA_TRY(cudaMemcpyAsync(staged + 3 * n, p.velocity, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, rest));
            CUDA_TRY(cudaMemcpyAsync(staged + 6 * n, p.mass, sizeof(float) * n, cudaMemcpyHostToDevice, rest));
            if (has_vol)
                CUDA_TRY(cudaMemcpyAsync(staged + 7 * n, p.volume, sizeof(float) * n, cudaMemcpyHostToDevice, rest));
            if (p.material)
                CUDA_TRY(cudaMemcpyAsync(staged_mat, p.material, sizeof(uint16_t) * n, cudaMemcpyHostToDevice, rest));
            if (sorted) CUDA_TRY(cudaEventRecord(compact_join_, compact_stream_));
            const uint32_t* perm = nullptr;
            DevMem sk[2], sv[2], sscr;  // back to the pool in the stream's order on return
            if (sorted) {
                SceneDev g{};
                sceneGeometry(*sc, 0, g);
                int bits = 1;
                while (((uint64_t)1 << bits) < ((uint64_t)sc->nblocks + 1) * 64) ++bits;
                for (int k = 0; k < 2; ++k) {
                    MPM_TRY(alloc(sk[k], sizeof(uint32_t) * n, "upload sort keys"));
                    MPM_TRY(alloc(sv[k], sizeof(uint32_t) * n, "upload sort values"));
                }
                MPM_TRY(alloc(sscr, sizeof(uint32_t) * onesweepScratchWords(n, bits), "upload sort scratch"));
                launchStagedKeys(stream_, num_sms_, g, staged, (uint32_t)n, sk[0].as<uint32_t>(), err_.as<uint32_t>());
                bool in_b = false;
                CUDA_TRY(radixSortOnesweep(sk[0].as<uint32_t>(), sv[0].as<uint32_t>(), sk[1].as<uint32_t>(),
                                           sv[1].as<uint32_t>(), n, bits, sscr.as<uint32_t>(), err_.as<uint32_t>(),
                                           &in_b, stream_));
                perm = sv[in_b ? 1 : 0].as<uint32_t>();
                CUDA_TRY(cudaStreamWaitEvent(stream_, compact_join_, 0));
            }
            const int b = parity_;
            launchInitState(stream_, num_sms_, sc->buf_f[b].as<float>(), sc->buf_pid[b].as<uint32_t>(),
                            sc->buf_mat[b].as<uint16_t>(), cap, staged, n, has_vol, perm, staged_mat);
            CUDA_TRY(cudaGetLastError());
            if (!p.material) CUDA_TRY(cudaMemsetAsync(sc->buf_mat[b].p, 0, sizeof(uint16_t) * n, stream_));
            // The caller's arrays may be freed once this returns.  Copies from
            // pageable memory have taken the data by then; copies from
            // page-locked memory are asynchronous, so wait for those only.
            if (anyPinned({p.position, p.velocity, p.mass, p.volume, p.material})) CUDA_TRY(cudaStreamSynchronize(stream_));
            drain.on = false;
        }
        sc->need_init = true;
        sc->stress_stale = true;
        *out_id = registerScene(std::move(sc));
        return MPM_OK;
    }

    // ---- checkpoints ----------------------------------------------------------
    // File layout (little endian): "MPMB200\0", u32 version, u32 sizeof(desc),
    // mpm_scene_desc, i32 nmaterials, mpm_material[nmaterials], u64 n,
    // u32 flags (bit 0: cached stress stale), then in the engine's internal
    // particle order the 41 float planes (n floats each), the original
    // particle ids (u32 x n) and the material ids (u16 x n); version 2 adds
    // u32 has_level_set and, if set, f32 friction, f32 velocity[3] and the
    // level set (f32 per grid node); version 3 adds f32 cfl, f64 simulated
    // time and f32 last dt; version 4 the semi-implicit settings f32 beta,
    // i32 max_iter, f32 tol.  Restoring that order and the cached stress
    // makes the continuation bitwise identical.  Older versions are still read.
    static constexpr uint32_t kCkptVersion = 4;

    mpm_status saveScene(int id, const char* path) {
        if (!path) return fail(MPM_ERR_INVALID_ARG, "null path");
        MPM_TRY(ensureReady());
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        SceneHost& s = *scenes_[idx];
        const size_t n = s.n;
        std::vector<float> planes((size_t)NFIELDS * n);
        std::vector<uint32_t> pid(n);
        std::vector<uint16_t> mat(n);
        CUDA_TRY(cudaStreamSynchronize(stream_));
        const size_t cap = std::max<size_t>(n, 1);
        for (int f = 0; f < NFIELDS && n; ++f)
            CUDA_TRY(cudaMemcpy(planes.data() + (size_t)f * n, s.buf_f[parity_].as<float>() + (size_t)f * cap,
                                sizeof(float) * n, cudaMemcpyDeviceToHost));
        if (n) {
            CUDA_TRY(cudaMemcpy(pid.data(), s.buf_pid[parity_].p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
            CUDA_TRY(cudaMemcpy(mat.data(), s.buf_mat[parity_].p, sizeof(uint16_t) * n, cudaMemcpyDeviceToHost));
        }
        std::vector<float> phi;
        if (s.has_phi) {
            phi.resize(s.nodes());
            CUDA_TRY(cudaMemcpy(phi.data(), s.phi.p, sizeof(float) * phi.size(), cudaMemcpyDeviceToHost));
        }
        const uint32_t has_phi = s.has_phi ? 1u : 0u;
        double sim_t = 0.0;
        float last_dt = 0.f;
        MPM_TRY(simTime(id, &sim_t, &last_dt));
        std::FILE* fp = std::fopen(path, "wb");
        if (!fp) return fail(MPM_ERR_IO, std::string("cannot open ") + path + " for writing");
        const char magic[8] = {'M', 'P', 'M', 'B', '2', '0', '0', 0};
        const uint32_t ver = kCkptVersion, dsz = (uint32_t)sizeof(mpm_scene_desc);
        const int32_t nm = (int32_t)s.mats_in.size();
        const uint64_t n64 = n;
        const uint32_t flags = s.stress_stale ? 1u : 0u;
        bool ok = std::fwrite(magic, 1, 8, fp) == 8 && std::fwrite(&ver, 4, 1, fp) == 1 &&
                  std::fwrite(&dsz, 4, 1, fp) == 1 && std::fwrite(&s.desc, sizeof(mpm_scene_desc), 1, fp) == 1 &&
                  std::fwrite(&nm, 4, 1, fp) == 1 &&
                  std::fwrite(s.mats_in.data(), sizeof(mpm_material), s.mats_in.size(), fp) == s.mats_in.size() &&
                  std::fwrite(&n64, 8, 1, fp) == 1 && std::fwrite(&flags, 4, 1, fp) == 1 &&
                  std::fwrite(planes.data(), sizeof(float), planes.size(), fp) == planes.size() &&
                  std::fwrite(pid.data(), sizeof(uint32_t), n, fp) == n &&
                  std::fwrite(mat.data(), sizeof(uint16_t), n, fp) == n && std::fwrite(&has_phi, 4, 1, fp) == 1;
        if (ok && has_phi)
            ok = std::fwrite(&s.phi_friction, 4, 1, fp) == 1 && std::fwrite(s.phi_vel, 4, 3, fp) == 3 &&
                 std::fwrite(phi.data(), sizeof(float), phi.size(), fp) == phi.size();
        ok = ok && std::fwrite(&s.cfl, 4, 1, fp) == 1 && std::fwrite(&sim_t, 8, 1, fp) == 1 &&
             std::fwrite(&last_dt, 4, 1, fp) == 1;
        ok = ok && std::fwrite(&s.beta, 4, 1, fp) == 1 && std::fwrite(&s.solve_max_iter, 4, 1, fp) == 1 &&
             std::fwrite(&s.solve_tol, 4, 1, fp) == 1;
        ok = (std::fclose(fp) == 0) && ok;
        if (!ok) return fail(MPM_ERR_IO, std::string("write failed: ") + path);
        return MPM_OK;
    }

    // Reads and checks a checkpoint on the host (no device work).
    struct Checkpoint {
        mpm_scene_desc desc{};
        std::vector<mpm_material> mats;
        size_t n = 0;
        uint32_t flags = 0;
        std::vector<float> planes;
        std::vector<uint32_t> pid;
        std::vector<uint16_t> mat;
        bool has_phi = false;
        float phi_friction = 0.f, phi_vel[3] = {0.f, 0.f, 0.f};
        std::vector<float> phi;
        float cfl = 0.f, last_dt = 0.f;
        double time = 0.0;
        float beta = 0.f, tol = 1e-5f;
        int32_t max_iter = 50;
    };
    static mpm_status readCheckpoint(const char* path, Checkpoint* ck) {
        if (!path) return fail(MPM_ERR_INVALID_ARG, "null path");
        std::FILE* fp = std::fopen(path, "rb");
        if (!fp) return fail(MPM_ERR_IO, std::string("cannot open ") + path);
        std::unique_ptr<std::FILE, int (*)(std::FILE*)> guard(fp, std::fclose);
        char magic[8];
        uint32_t ver = 0, dsz = 0;
        int32_t nm = 0;
        uint64_t n64 = 0;
        if (std::fread(magic, 1, 8, fp) != 8 || memcmp(magic, "MPMB200", 8) != 0)
            return fail(MPM_ERR_PARSE, std::string(path) + ": not a checkpoint");
        if (std::fread(&ver, 4, 1, fp) != 1 || ver < 1 || ver > kCkptVersion || std::fread(&dsz, 4, 1, fp) != 1 ||
            dsz != sizeof(mpm_scene_desc))
            return fail(MPM_ERR_PARSE, std::string(path) + ": unsupported checkpoint version");
        if (std::fread(&ck->desc, sizeof(mpm_scene_desc), 1, fp) != 1 || std::fread(&nm, 4, 1, fp) != 1 || nm < 1 ||
            nm > 65535)
            return fail(MPM_ERR_PARSE, std::string(path) + ": truncated or corrupt header");
        ck->mats.resize(nm);
        if (std::fread(ck->mats.data(), sizeof(mpm_material), nm, fp) != (size_t)nm ||
            std::fread(&n64, 8, 1, fp) != 1 || n64 > 0x7fffffffull || std::fread(&ck->flags, 4, 1, fp) != 1)
            return fail(MPM_ERR_PARSE, std::string(path) + ": truncated or corrupt header");
        mpm_particles_in none{};
        none.materials = ck->mats.data();
        none.nmaterials = nm;
        MPM_TRY(validate(ck->desc, none));
        const size_t n = (size_t)n64;
        ck->n = n;
        try {
            ck->planes.resize((size_t)NFIELDS * n);
            ck->pid.resize(n);
            ck->mat.resize(n);
        } catch (const std::bad_alloc&) {
            return fail(MPM_ERR_OOM, "host allocation failed");
        }
        if (std::fread(ck->planes.data(), sizeof(float), ck->planes.size(), fp) != ck->planes.size() ||
            std::fread(ck->pid.data(), sizeof(uint32_t), n, fp) != n ||
            std::fread(ck->mat.data(), sizeof(uint16_t), n, fp) != n)
            return fail(MPM_ERR_PARSE, std::string(path) + ": truncated particle data");
        if (ver >= 2) {
            uint32_t has_phi = 0;
            if (std::fread(&has_phi, 4, 1, fp) != 1 || has_phi > 1)
                return fail(MPM_ERR_PARSE, std::string(path) + ": truncated or corrupt level-set section");
            if (has_phi) {
                const size_t nodes = (size_t)ck->desc.resolution[0] * ck->desc.resolution[1] * ck->desc.resolution[2];
                try {
                    ck->phi.resize(nodes);
                } catch (const std::bad_alloc&) {
                    return fail(MPM_ERR_OOM, "host allocation failed");
                }
                if (std::fread(&ck->phi_friction, 4, 1, fp) != 1 || std::fread(ck->phi_vel, 4, 3, fp) != 3 ||
                    std::fread(ck->phi.data(), sizeof(float), nodes, fp) != nodes)
                    return fail(MPM_ERR_PARSE, std::string(path) + ": truncated level-set section");
                ck->has_phi = true;
            }
        }
        if (ver >= 3) {
            if (std::fread(&ck->cfl, 4, 1, fp) != 1 || std::fread(&ck->time, 8, 1, fp) != 1 ||
                std::fread(&ck->last_dt, 4, 1, fp) != 1 || !(ck->cfl >= 0.f) || !std::isfinite(ck->cfl))
                return fail(MPM_ERR_PARSE, std::string(path) + ": truncated or corrupt time section");
        }
        if (ver >= 4) {
            if (std::fread(&ck->beta, 4, 1, fp) != 1 || std::fread(&ck->max_iter, 4, 1, fp) != 1 ||
                std::fread(&ck->tol, 4, 1, fp) != 1)
                return fail(MPM_ERR_PARSE, std::string(path) + ": truncated solver section");
        }
        std::vector<uint8_t> seen(n, 0);
        for (size_t i = 0; i < n; ++i) {
            if (ck->pid[i] >= n || seen[ck->pid[i]]) return fail(MPM_ERR_PARSE, std::string(path) + ": bad particle ids");
            seen[ck->pid[i]] = 1;
            if (ck->mat[i] >= (uint32_t)nm) return fail(MPM_ERR_PARSE, std::string(path) + ": bad material ids");
        }
        return MPM_OK;
    }

    mpm_status loadScene(const Checkpoint& ck, int* out_id) {
        std::unique_ptr<SceneHost> sc;
        MPM_TRY(newScene(ck.desc, ck.mats.data(), (int)ck.mats.size(), ck.n, &sc));
        const size_t n = ck.n, cap = std::max<size_t>(n, 1);
        const int b = parity_;
        for (int f = 0; f < NFIELDS && n; ++f)
            CUDA_TRY(cudaMemcpyAsync(sc->buf_f[b].as<float>() + (size_t)f * cap, ck.planes.data() + (size_t)f * n,
                                     sizeof(float) * n, cudaMemcpyHostToDevice, stream_));
        if (n) {
            CUDA_TRY(cudaMemcpyAsync(sc->buf_pid[b].p, ck.pid.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice,
                                     stream_));
            CUDA_TRY(cudaMemcpyAsync(sc->buf_mat[b].p, ck.mat.data(), sizeof(uint16_t) * n, cudaMemcpyHostToDevice,
                                     stream_));
        }
        CUDA_TRY(cudaStreamSynchronize(stream_));
        sc->need_init = false;  // V0 is part of the state
        sc->stress_stale = (ck.flags & 1u) != 0;
        sc->time_fixed = ck.time;
        sc->last_dt = ck.last_dt;
        sc->cfl = ck.cfl;
        *out_id = registerScene(std::move(sc));
        if (ck.has_phi) {
            mpm_status st = setLevelSet(*out_id, ck.phi.data(), ck.phi_friction, ck.phi_vel);
            if (st != MPM_OK) {
                removeScene(*out_id);
                return st;
            }
        }
        if (ck.beta > 0.f) {
            mpm_status st = setImplicit(*out_id, ck.beta, ck.max_iter, ck.tol);
            if (st != MPM_OK) {
                removeScene(*out_id);
                return st;
            }
        }
        return MPM_OK;
    }

    mpm_status removeScene(int id) {
        for (size_t i = 0; i < scenes_.size(); ++i)
            if (scenes_[i]->id == id) {
                // Its device memory returns to the pool in stream order (after
                // the queued steps), so the host does not wait here.
                scenes_.erase(scenes_.begin() + i);
                dirty_ = true;
                keys_valid_ = false;
                sorted_valid_ = false;
                return MPM_OK;
            }
        return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
    }

    SceneHost* scene(int id) {
        for (auto& s : scenes_)
            if (s->id == id) return s.get();
        return nullptr;
    }
    int sceneIndex(int id) const {
        for (size_t i = 0; i < scenes_.size(); ++i)
            if (scenes_[i]->id == id) return (int)i;
        return -1;
    }

    // Rebuild the device scene table and the batch-wide scratch after the
    // set of scenes changed.
    // The grid geometry of a scene's table entry (what its cell keys need),
    // with its blocks numbered from block_base.
    static void sceneGeometry(const SceneHost& s, uint32_t block_base, SceneDev& d) {
        for (int a = 0; a < 3; ++a) {
            d.origin[a] = s.desc.origin[a];
            d.res[a] = s.desc.resolution[a];
            d.nb[a] = s.nb[a];
            d.target[a] = s.desc.origin[a] + s.desc.stride * (float)s.desc.resolution[a];
        }
        d.h = s.desc.stride;
        d.inv_h = 1.0f / s.desc.stride;
        d.range = stencilRange(s.desc.interpolation);
        d.block_base = block_base;
        d.nblocks = s.nblocks;
        d.S = s.S;
    }

    mpm_status rebuild() {
        if (!dirty_) return MPM_OK;
        CUDA_TRY(cudaStreamSynchronize(stream_));
        dropGraphs();  // graphs hold pointers into buffers that may move below
        const int ns = (int)scenes_.size();
        host_scenes_.assign(ns, SceneDev{});
        std::vector<uint32_t> sbb(ns + 1, 0);
        size_t ntot = 0;
        uint64_t tb = 0;
        max_nodes_ = 0;
        max_n_ = 0;
        for (int i = 0; i < ns; ++i) {
            SceneHost& s = *scenes_[i];
            SceneDev& d = host_scenes_[i];
            sceneGeometry(s, (uint32_t)tb, d);
            sbb[i] = (uint32_t)tb;
            tb += (uint64_t)s.nblocks + 1;  // + the scene's outside block
            d.key_offset = (uint32_t)ntot;
            d.n = (uint32_t)s.n;
            d.cap = (uint32_t)std::max<size_t>(s.n, 1);
            ntot += s.n;
            d.dt = s.desc.dt;
            d.gravity = s.desc.gravity;
            d.friction = s.desc.friction;
            d.blend = s.desc.blend;
            d.dinv = 0.f;
            if (s.desc.transfer == MPM_TRANSFER_APIC) {
                // D = k h^2 I, k = 1/3 cubic, 1/4 quadratic (src/apic_mpm_solver3d.cu:151-157)
                float k = s.desc.interpolation == MPM_INTERP_CUBIC_BSPLINE ? (float)(1 / 3.0) : (float)(1 / 4.0);
                d.dinv = 1.0f / (k * s.desc.stride * s.desc.stride);
            }
            d.transfer = s.desc.transfer;
            d.interp = s.desc.interpolation;
            d.combo = comboIndex(s.S, s.desc.transfer);
            d.boundary = s.desc.boundary;
            d.sticky = s.desc.sticky_cells;
            d.pcoll = s.desc.particles_collision;
            d.nmat = s.nmat;
            for (int b = 0; b < 2; ++b) {
                d.buf[b].f = s.buf_f[b].as<float>();
                d.buf[b].pid = s.buf_pid[b].as<uint32_t>();
                d.buf[b].mat = s.buf_mat[b].as<uint16_t>();
            }
            d.vstar = s.vstar.as<float4>();
            d.vold = s.vold.as<float4>();
            d.mats = s.mats.as<MaterialDev>();
            d.dbg = s.dbg.as<float>();
            d.phi = s.has_phi ? s.phi.as<float>() : nullptr;
            d.phi_friction = s.phi_friction;
            for (int a = 0; a < 3; ++a) d.phi_vel[a] = s.phi_vel[a];
            d.cfl = s.cfl;
            d.dt_max = s.desc.dt;
            d.cfl_state = s.cfl_state.as<CflState>();
            solveFields(s, d);
            max_nodes_ = std::max(max_nodes_, s.nodes());
            max_n_ = std::max(max_n_, s.n);
        }
        sbb[ns] = (uint32_t)tb;
        any_cfl_ = false;
        for (auto& s : scenes_) any_cfl_ |= s->cfl > 0.f;
        if (tb * 64 > 0xffffffffull) return fail(MPM_ERR_UNSUPPORTED, "batch grid too large for 32-bit cell keys");
        if (ntot > 0x7fffffffull) return fail(MPM_ERR_UNSUPPORTED, "batch has too many particles");
        ntot_ = ntot;
        total_blocks_ = (uint32_t)tb;
        key_bits_ = 1;
        while (((uint64_t)1 << key_bits_) < tb * 64) ++key_bits_;
        // batch scratch
        const size_t nk = std::max<size_t>(ntot, 1);
        for (int k = 0; k < 2; ++k) {
            MPM_TRY(grow(keys_[k], sizeof(uint32_t) * nk, "keys"));
            MPM_TRY(grow(vals_[k], sizeof(uint32_t) * nk, "values"));
        }
        MPM_TRY(grow(sort_scratch_, sizeof(uint32_t) * onesweepScratchWords(nk, key_bits_), "sort scratch"));
        MPM_TRY(grow(inc_scratch_, sizeof(uint32_t) * incrementalSortScratchWords(nk, key_bits_),
                                  "incremental sort scratch"));
        MPM_TRY(grow(compact_scratch_, sizeof(unsigned long long) * compactScratchWords64((uint32_t)tb),
                                       "compaction scratch"));
        MPM_TRY(grow(block_count_, sizeof(uint32_t) * tb, "block counts"));
        CUDA_TRY(cudaMemsetAsync(block_count_.p, 0, sizeof(uint32_t) * tb, stream_));
        MPM_TRY(grow(sbb_, sizeof(uint32_t) * (ns + 1), "scene block bases"));
        CUDA_TRY(cudaMemcpyAsync(sbb_.p, sbb.data(), sizeof(uint32_t) * (ns + 1), cudaMemcpyHostToDevice, stream_));
        // work items: one per non-empty block plus one per further kBlockChunk particles
        max_active_ = std::max<size_t>(1, std::min<size_t>(tb, nk) + nk / kBlockChunk + 1);
        MPM_TRY(grow(active_, sizeof(BlockItem) * max_active_, "active blocks"));
        MPM_TRY(grow(outside_, sizeof(BlockItem) * ((size_t)ns + nk / kBlockChunk + 1), "outside blocks"));
        g2p_cap_ = (uint32_t)(std::min<size_t>(tb, nk) + nk / kMinG2PChunk + 1);
        MPM_TRY(grow(g2p_items_, sizeof(BlockItem) * g2p_cap_ * (size_t)combos().size(), "G2P items"));
        // P2G's two lists of item slots per combination (warp items, CTA items)
        MPM_TRY(grow(p2g_lists_, sizeof(uint32_t) * max_active_ * 2 * combos().size(), "P2G item lists"));
        // [0] work items, [1] outside items, [2] active nodes, [8 + 8k .. 13 + 8k] item
        // schedulers of the k-th stencil/transfer combination, then the G2P
        // item counts (kG2PCountWord) and the P2G list counts (kP2GListWord)
        MPM_TRY(alloc(counters_, sizeof(uint32_t) * kCounterWords, "counters"));
        if (!spans_.p) {
            MPM_TRY(alloc(spans_, sizeof(unsigned long long) * kSpanWords * kMaxCombos, "kernel spans"));
            MPM_TRY(resetSpans());
        }
        CUDA_TRY(cudaMemsetAsync(counters_.p, 0, sizeof(uint32_t) * kCounterWords, stream_));
        MPM_TRY(grow(block_slot_, sizeof(int32_t) * tb, "block slots"));
        int maxS = 2;
        for (auto& s : scenes_) maxS = std::max(maxS, s->S);
        tile_stride_ = (size_t)7 * tileNodes(maxS);
        MPM_TRY(grow(tiles_, sizeof(float) * tile_stride_ * max_active_, "P2G tiles"));
        MPM_TRY(grow(scenes_dev_, sizeof(SceneDev) * std::max(ns, 1), "scene table"));
        // Room in the pool for the download staging buffers (two float4 per
        // particle, taken at a scene's first download): taken and given back
        // here, so that the first download -- or a later engine's -- finds the
        // memory in the pool instead of growing it in the middle of a run
        // (about 1 ms for a 1M-particle scene).  Best effort.
        if (ntot > staging_reserved_) {
            void* p = nullptr;
            if (cudaMallocFromPoolAsync(&p, (size_t)32 * ntot, pool_, stream_) == cudaSuccess) {
                CUDA_TRY(cudaFreeAsync(p, stream_));
                staging_reserved_ = ntot;
            } else {
                cudaGetLastError();
            }
        }
        // TMA maps of each scene's v* and v grids (G2P stages its tiles with them)
        {
            std::vector<unsigned char> maps((size_t)2 * kTensorMapBytes * std::max(ns, 1), 0);
            for (int i = 0; i < ns; ++i) {
                const SceneDev& d = host_scenes_[i];
                const int T = d.S + 3;
                const char* e1 = encodeGridTensorMap(maps.data() + (size_t)2 * i * kTensorMapBytes, d.vstar, d.res, T);
                const char* e2 = encodeGridTensorMap(maps.data() + (size_t)(2 * i + 1) * kTensorMapBytes,
                                                     d.vold ? (const void*)d.vold : (const void*)d.vstar, d.res, T);
                if (e1 || e2) return fail(MPM_ERR_CUDA, std::string("grid tensor map: ") + (e1 ? e1 : e2));
            }
            MPM_TRY(grow(tmaps_, maps.size(), "grid tensor maps"));
            if (((uintptr_t)tmaps_.p & 63u) != 0) return fail(MPM_ERR_CUDA, "tensor map table not 64-byte aligned");
            CUDA_TRY(cudaMemcpyAsync(tmaps_.p, maps.data(), maps.size(), cudaMemcpyHostToDevice, stream_));
            CUDA_TRY(cudaStreamSynchronize(stream_));  // the host table is freed on return
        }
        CUDA_TRY(cudaMemcpyAsync(scenes_dev_.p, host_scenes_.data(), sizeof(SceneDev) * ns, cudaMemcpyHostToDevice,
                                 stream_));
        CUDA_TRY(cudaStreamSynchronize(stream_));
        kcur_ = 0;
        dirty_ = false;
        keys_valid_ = false;
        sorted_valid_ = false;
        incremental_ok_ = false;
        stage_check_ = true;
        stage_pending_ = false;  // a read-back issued before the sync above is stale
        for (bool& f : warp_few_) f = false;  // the new set's small items: decided on the device until read back
        any_implicit_ = false;
        for (auto& s : scenes_) any_implicit_ |= s->beta > 0.f;
        MPM_TRY(ensureSolveBuffers());
        return MPM_OK;
    }

    // ---- semi-implicit update ---------------------------------------------
    static void solveFields(const SceneHost& s, SceneDev& d) {
        d.beta = s.beta;
        d.solve_tol = s.solve_tol;
        d.solve_max_iter = s.solve_max_iter;
        d.solve = SolveDev{s.solve_m.as<float>(), s.solve_vec.as<float4>(), s.solve_list.as<int>(),
                           s.solve_part.as<double>(), s.solve_status.as<SolveStatus>()};
    }
    // Batch-wide buffers over the sorted particles and the cell keys.
    mpm_status ensureSolveBuffers() {
        if (!any_implicit_ || dirty_) return MPM_OK;
        const size_t n = std::max<size_t>(ntot_, 1);
        MPM_TRY(grow(cell_range_, sizeof(uint2) * (size_t)total_blocks_ * 64, "solver cell ranges"));
        MPM_TRY(grow(block_range_, sizeof(uint2) * (size_t)total_blocks_, "solver block ranges"));
        MPM_TRY(grow(solve_pofs_, sizeof(float4) * n, "solver stencil offsets"));
        MPM_TRY(grow(solve_prep_, sizeof(float) * kSolvePrepPlanes * n, "solver particle data"));
        MPM_TRY(grow(solve_T_, sizeof(float4) * 3 * n, "solver particle stress differentials"));
        MPM_TRY(grow(solve_iter_, sizeof(int), "solver iteration counter"));
        MPM_TRY(ensureSideStreams(1));  // the loop body of a captured solve is captured on side_[0]
        return MPM_OK;
    }
    // beta > 0: every step solves (M + beta dt^2 H) v = M v* after the grid
    // collision (beta 1/2: Crank-Nicolson-like, 1: backward Euler), to
    // |r| <= tol |M v*| or max_iter iterations; beta = 0: explicit.
    mpm_status setImplicit(int id, float beta, int max_iter, float tol) {
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        if (!(beta >= 0.f) || !std::isfinite(beta)) return fail(MPM_ERR_INVALID_ARG, "beta must be finite and >= 0");
        if (max_iter < 1 || max_iter > 10000) return fail(MPM_ERR_INVALID_ARG, "max_iter must be in [1, 10000]");
        if (!(tol >= 0.f) || !std::isfinite(tol)) return fail(MPM_ERR_INVALID_ARG, "tol must be finite and >= 0");
        CUDA_TRY(cudaStreamSynchronize(stream_));
        SceneHost& s = *scenes_[idx];
        if (beta > 0.f) {
            const size_t nodes = s.nodes();
            MPM_TRY(grow(s.solve_m, sizeof(float) * nodes, "solver node masses"));
            MPM_TRY(grow(s.solve_vec, sizeof(float4) * kSolveVectors * nodes, "solver node vectors"));
            MPM_TRY(grow(s.solve_list, sizeof(int) * nodes, "solver node list"));
            MPM_TRY(grow(s.solve_part, sizeof(double) * solvePartialDoubles(max_iter), "solver partial sums"));
            MPM_TRY(grow(s.solve_status, sizeof(SolveStatus), "solver status"));
            CUDA_TRY(cudaMemset(s.solve_status.p, 0, sizeof(SolveStatus)));
        }
        s.beta = beta;
        s.solve_max_iter = max_iter;
        s.solve_tol = tol;
        dropGraphs();  // the launch sequence depends on the solver settings
        any_implicit_ = false;
        for (auto& sc : scenes_) any_implicit_ |= sc->beta > 0.f;
        if (!dirty_) {
            solveFields(s, host_scenes_[idx]);
            MPM_TRY(ensureSolveBuffers());
            MPM_TRY(uploadSceneTable());
        }
        return MPM_OK;
    }
    mpm_status solveInfo(int id, int* iters, float* residual) {
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        SolveStatus st{};
        CUDA_TRY(cudaStreamSynchronize(stream_));
        if (scenes_[idx]->solve_status.p)
            CUDA_TRY(cudaMemcpy(&st, scenes_[idx]->solve_status.p, sizeof(SolveStatus), cudaMemcpyDeviceToHost));
        if (iters) *iters = st.iters;
        if (residual) *residual = st.residual;
        return MPM_OK;
    }
    int maxSolveIters() const {
        int m = 0;
        for (auto& s : scenes_)
            if (s->beta > 0.f) m = std::max(m, s->solve_max_iter);
        return m;
    }
    mpm_status launchSolveAll(bool split) {
        SolveBuffers b{keys_[sorted_].as<uint32_t>(), vals_[sorted_].as<uint32_t>(), cell_range_.as<uint2>(),
                       (size_t)total_blocks_ * 64, block_range_.as<uint2>(), (size_t)total_blocks_,
                       solve_pofs_.as<float4>(), solve_prep_.as<float>(), solve_T_.as<float4>(), (uint32_t)ntot_,
                       solve_iter_.as<int>()};
        const std::vector<int> S = stencilSizes();
        CUDA_TRY(launchSolve(ctx(), b, parity_, S.data(), (int)S.size(), maxSolveIters(), split, side_[0]));
        return MPM_OK;
    }
    // Split API: solveLinearSystem(dt) on the split-mode grid (v* of
    // updateGridVelocities / gridCollision), no collision after.
    mpm_status solveLinearSystem(float dt) {
        MPM_TRY(ensureReady());
        if (!any_implicit_) return MPM_OK;  // explicit: the reference's no-op
        MPM_TRY(ensureDbg());
        if (!sorted_valid_) MPM_TRY(sortLive());
        std::vector<SceneDev> saved = host_scenes_;
        for (auto& d : host_scenes_) d.dt = dt;
        MPM_TRY(uploadSceneTable());
        MPM_TRY(launchSolveAll(true));
        host_scenes_ = saved;
        MPM_TRY(uploadSceneTable());
        return MPM_OK;
    }

    mpm_status uploadSceneTable() {
        CUDA_TRY(cudaMemcpyAsync(scenes_dev_.p, host_scenes_.data(), sizeof(SceneDev) * host_scenes_.size(),
                                 cudaMemcpyHostToDevice, stream_));
        return MPM_OK;
    }

    LaunchCtx ctx() const {
        LaunchCtx c;
        c.scenes = scenes_dev_.as<SceneDev>();
        c.nscenes = (int)scenes_.size();
        c.stream = stream_;
        c.num_sms = num_sms_;
        c.p2g_stage = p2g_stage_;
        c.particle_blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((max_n_ + kThreads - 1) / kThreads,
                                                                           (size_t)num_sms_ * 16));
        c.node_blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((max_nodes_ + kThreads - 1) / kThreads,
                                                                       (size_t)num_sms_ * 16));
        c.persistent_blocks = (unsigned)std::max<size_t>(1, std::min<size_t>(max_active_ + 64, (size_t)num_sms_ * 4));
        return c;
    }

    StepArgs args(const uint32_t* sorted_keys, const uint32_t* perm, uint32_t* next_keys) const {
        StepArgs a;
        a.scenes = scenes_dev_.as<SceneDev>();
        a.nscenes = (int)scenes_.size();
        a.parity = parity_;
        a.sorted_keys = sorted_keys;
        a.perm = perm;
        a.active = active_.as<BlockItem>();
        a.g2p_items = g2p_items_.as<BlockItem>();
        a.g2p_cap = g2p_cap_;
        a.combo = 0;
        a.counters = counters_.as<uint32_t>();
        a.outside = outside_.as<BlockItem>();
        a.block_slot = block_slot_.as<int32_t>();
        a.tiles = tiles_.as<float>();
        a.tile_stride = (uint32_t)tile_stride_;
        a.next_keys = next_keys;
        a.block_count = block_count_.as<uint32_t>();
        a.err = err_.as<uint32_t>();
        a.stats = counters_.as<uint32_t>();
        a.sched = counters_.as<uint32_t>() + 8;
        a.tmaps = tmaps_.as<unsigned char>();
        a.spans = nullptr;  // set per combination by the step
        a.p2g_lists = nullptr;  // the step's P2G launches take their combination's lists
        a.p2g_list_cap = (uint32_t)max_active_;
        a.p2g_warp = P2G_WARP_NONE;
        return a;
    }

    BlockBuffers blockBuffers() const {
        BlockBuffers bb;
        bb.block_count = block_count_.as<uint32_t>();
        bb.scene_block_base = sbb_.as<uint32_t>();
        bb.active = active_.as<BlockItem>();
        bb.outside = outside_.as<BlockItem>();
        bb.g2p_items = g2p_items_.as<BlockItem>();
        bb.g2p_cap = g2p_cap_;
        bb.counters = counters_.as<uint32_t>();
        bb.block_slot = block_slot_.as<int32_t>();
        bb.p2g_lists = p2g_lists_.as<uint32_t>();
        bb.p2g_list_cap = (uint32_t)max_active_;
        return bb;
    }

    // Profiling: an event pair per kernel family launch, recorded on the
    // engine's stream without synchronizing; resolved in accumulateProfile().
    cudaEvent_t takeEvent() {
        cudaEvent_t e = nullptr;
        if (!event_pool_.empty()) {
            e = event_pool_.back();
            event_pool_.pop_back();
        } else if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            e = nullptr;
        }
        return e;
    }
    void mark(int fam, int which) {
        if (!profiling_) return;
        if (which == 0) {
            open_[fam] = takeEvent();
            if (open_[fam]) cudaEventRecord(open_[fam], stream_);
        } else if (open_[fam]) {
            cudaEvent_t e1 = takeEvent();
            if (e1) {
                cudaEventRecord(e1, stream_);
                records_.push_back({fam, open_[fam], e1});
            } else {
                event_pool_.push_back(open_[fam]);
            }
            open_[fam] = nullptr;
        }
    }
    void collect(int) {}

    // Keys of the live order (if stale) + sort + compaction.
    mpm_status sortLive() {
        if (!keys_valid_) {
            mark(KF_KEYS, 0);
            CUDA_TRY(cudaMemsetAsync(block_count_.p, 0, sizeof(uint32_t) * total_blocks_, stream_));
            launchKeys(ctx(), parity_, keys_[kcur_].as<uint32_t>(), block_count_.as<uint32_t>(), err_.as<uint32_t>());
            mark(KF_KEYS, 1);
            collect(KF_KEYS);
            keys_valid_ = true;
        }
        const bool incremental =
            incremental_ok_ && !full_sort_only_ && (ntot_ >= kIncrementalMinKeys || incremental_always_);
        // The block compaction reads only the per-block counts, not the sorted
        // keys: beside the full radix sort (both latency-bound) it runs on its
        // own stream and joins before the caller's next launch (two-ball step
        // 0.425 -> 0.418 ms).  Beside the incremental sort it costs more than
        // it hides (64-scene batch 2.34 -> 2.38 ms), and profiling keeps the
        // families in sequence so that each is timed alone.
        const bool overlap = !profiling_ && !incremental;
        if (overlap) {
            CUDA_TRY(cudaEventRecord(compact_fork_, stream_));
            CUDA_TRY(cudaStreamWaitEvent(compact_stream_, compact_fork_, 0));
            LaunchCtx cc = ctx();
            cc.stream = compact_stream_;
            launchCompactOnesweep(cc, blockBuffers(), total_blocks_, compact_scratch_.as<unsigned long long>(), kBlockChunk, comboSplit(),
                                  err_.as<uint32_t>());
            CUDA_TRY(cudaGetLastError());
            CUDA_TRY(cudaEventRecord(compact_join_, compact_stream_));
        }
        mark(KF_SORT, 0);
        if (incremental) {
            // keys_[1 - kcur_] still holds the previous step's sorted keys,
            // aligned with the live particle order: sort incrementally into it
            const int out = 1 - kcur_;
            CUDA_TRY(incrementalSort(keys_[kcur_].as<uint32_t>(), keys_[out].as<uint32_t>(), ntot_, key_bits_,
                                     keys_[out].as<uint32_t>(), vals_[out].as<uint32_t>(), inc_scratch_.as<uint32_t>(),
                                     err_.as<uint32_t>(), stream_));
            sorted_ = out;
        } else {
            bool inB = false;
            CUDA_TRY(radixSortOnesweep(keys_[kcur_].as<uint32_t>(), vals_[kcur_].as<uint32_t>(),
                                       keys_[1 - kcur_].as<uint32_t>(), vals_[1 - kcur_].as<uint32_t>(), ntot_,
                                       key_bits_, sort_scratch_.as<uint32_t>(), err_.as<uint32_t>(), &inB, stream_));
            sorted_ = inB ? 1 - kcur_ : kcur_;
        }
        incremental_ok_ = false;  // set again once G2P has reordered the particles by this sort
        mark(KF_SORT, 1);
        collect(KF_SORT);
        if (overlap) {
            CUDA_TRY(cudaStreamWaitEvent(stream_, compact_join_, 0));
        } else {
            mark(KF_COMPACT, 0);
            launchCompactOnesweep(ctx(), blockBuffers(), total_blocks_, compact_scratch_.as<unsigned long long>(), kBlockChunk, comboSplit(),
                                  err_.as<uint32_t>());
            mark(KF_COMPACT, 1);
            collect(KF_COMPACT);
        }
        CUDA_TRY(cudaGetLastError());
        sorted_valid_ = true;
        return MPM_OK;
    }

    struct Combo {
        int S;
        int transfer;
    };
    std::vector<Combo> combos() const {
        std::vector<Combo> c;
        for (auto& s : scenes_) {
            bool found = false;
            for (auto& e : c)
                if (e.S == s->S && e.transfer == s->desc.transfer) found = true;
            if (!found) c.push_back({s->S, s->desc.transfer});
        }
        return c;
    }
    int comboIndex(int S, int transfer) const {
        auto cs = combos();
        for (size_t k = 0; k < cs.size(); ++k)
            if (cs[k].S == S && cs[k].transfer == transfer) return (int)k;
        return 0;
    }
    std::vector<int> stencilSizes() const {
        std::vector<int> v;
        for (auto& s : scenes_)
            if (std::find(v.begin(), v.end(), s->S) == v.end()) v.push_back(s->S);
        return v;
    }

    mpm_status ensureReady() {
        if (scenes_.empty()) return fail(MPM_ERR_INVALID_ARG, "no scenes");
        MPM_TRY(rebuild());
        bool need = false;
        for (auto& s : scenes_) need |= s->need_init;
        if (need) MPM_TRY(initialize(false));
        return MPM_OK;
    }

    // initialize(): V0 from the grid mass (src/mpm_solver3d.cu:131-223).
    mpm_status initialize(bool all) {
        MPM_TRY(rebuild());
        bool any_estimate = false;
        for (auto& s : scenes_)
            if ((all || s->need_init) && s->desc.volume_mode == MPM_VOLUME_GRID_ESTIMATE) any_estimate = true;
        if (any_estimate) {
            // the mass pass covers only the scenes being initialized
            for (size_t i = 0; i < scenes_.size(); ++i)
                host_scenes_[i].init_pass = (all || scenes_[i]->need_init) ? 1 : 0;
            MPM_TRY(uploadSceneTable());
            MPM_TRY(sortLive());
            StepArgs a = args(keys_[sorted_].as<uint32_t>(), vals_[sorted_].as<uint32_t>(), nullptr);
            LaunchCtx c = ctx();
            for (int S : stencilSizes()) {
                launchP2G(c, a, S, MODE_MASS, -1);
                launchGrid(c, a, S, MODE_MASS, -1);
            }
            // The volume kernel runs per scene so that only scenes being
            // initialized get a new V0.
            for (size_t i = 0; i < scenes_.size(); ++i) {
                SceneHost& s = *scenes_[i];
                if (!(all || s.need_init) || s.desc.volume_mode != MPM_VOLUME_GRID_ESTIMATE) continue;
                LaunchCtx one = c;
                one.scenes = scenes_dev_.as<SceneDev>() + i;
                one.nscenes = 1;
                launchVolume(one, parity_, s.S);
            }
            CUDA_TRY(cudaGetLastError());
            // The sort and the work items stay valid for the first step (the
            // positions have not moved); the block counts were consumed by the
            // compaction, so the keys must be recounted after that step.
            keys_valid_ = false;
        }
        for (auto& s : scenes_) {
            if (all || s->need_init) s->stress_stale = true;  // V0 changed
            s->need_init = false;
        }
        return MPM_OK;
    }

    // tau from Fe/Fp for the scenes whose cached stress is stale (new scenes,
    // uploads, re-initialization).  Scenes whose tau came from the last G2P
    // keep it, so a scene's trajectory does not depend on its batch-mates.
    mpm_status refreshStress() {
        bool any = false;
        for (auto& s : scenes_) any |= s->stress_stale;
        if (!any) return MPM_OK;
        mark(KF_STRESS, 0);
        LaunchCtx c = ctx();
        for (size_t i = 0; i < scenes_.size(); ++i) {
            if (!scenes_[i]->stress_stale) continue;
            LaunchCtx one = c;
            one.scenes = scenes_dev_.as<SceneDev>() + i;
            one.nscenes = 1;
            launchStress(one, parity_);
            scenes_[i]->stress_stale = false;
        }
        mark(KF_STRESS, 1);
        CUDA_TRY(cudaGetLastError());
        return MPM_OK;
    }

    // One fused simulateOneStep over every scene of the batch.  In steady state
    // (keys and stress produced by the previous G2P, no profiling) the step is
    // replayed from a CUDA graph captured once per (particle buffer, key
    // buffer) state; the launch sequence and its arguments only depend on it.
    bool steadyNow() const {
        bool stale = false;
        for (auto& s : scenes_) stale |= s->stress_stale;
        return use_graphs_ && keys_valid_ && incremental_ok_ && !stale && !profiling_ && !dirty_ && !stage_check_ &&
               !tune_run_;
    }

    // Captures the step of the current host state into g (the host state is
    // left as it was: the capture only records the launches).  On a capture
    // failure graphs are switched off for this engine and g stays empty.
    mpm_status captureGraph(GraphSlot& g) {
        const int p0 = parity_, k0 = kcur_;
        const uint64_t l0 = kernelLaunches();
        sorted_valid_ = false;  // the graph must contain the sort
        CUDA_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        mpm_status st = stepBody();
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream_, &graph);
        parity_ = p0;
        kcur_ = k0;
        keys_valid_ = true;
        if (st == MPM_OK && e == cudaSuccess) {
            e = cudaGraphInstantiate(&g.exec, graph, 0);
            if (e != cudaSuccess) g.exec = nullptr;
        }
        if (graph) cudaGraphDestroy(graph);
        if (st != MPM_OK || e != cudaSuccess) {
            cudaGetLastError();
            use_graphs_ = false;  // fall back to direct launches for this engine
            noteLaunches(0 - (kernelLaunches() - l0));
            return MPM_OK;
        }
        g.launches = kernelLaunches() - l0;
        noteLaunches(0 - g.launches);  // captured, not run: counted at each replay instead
        return MPM_OK;
    }

    // Host state after a replayed step of the state (p0, k0), as stepBody()
    // leaves it.
    void advanceReplayed(int p0, int k0) {
        sorted_ = graph_sorted_[p0][k0];
        parity_ = p0 ^ 1;
        kcur_ = 1 - sorted_;
        keys_valid_ = true;
        sorted_valid_ = false;
        incremental_ok_ = true;
    }

    // Captures, ahead of time, the graphs of the states the next steps visit
    // (they alternate between particle buffers and key buffers), so that a
    // timed run replays graphs from its first step instead of capturing inside
    // its timed region.  Resolves a pending staging decision first.
    mpm_status prepareGraphs() {
        if (stage_pending_) {
            CUDA_TRY(cudaEventSynchronize(stage_event_));
            MPM_TRY(checkP2GStage());
        }
        const int p0 = parity_, k0 = kcur_, s0 = sorted_;
        const bool kv = keys_valid_, sv = sorted_valid_, io = incremental_ok_;
        for (int i = 0; i < 4 && steadyNow(); ++i) {
            GraphSlot& g = graphs_[parity_][kcur_];
            if (!g.exec) MPM_TRY(captureGraph(g));
            if (!g.exec) break;
            advanceReplayed(parity_, kcur_);
        }
        parity_ = p0;
        kcur_ = k0;
        sorted_ = s0;
        keys_valid_ = kv;
        sorted_valid_ = sv;
        incremental_ok_ = io;
        return MPM_OK;
    }

    // One fused simulateOneStep over every scene of the batch.  In steady state
    // (keys and stress produced by the previous G2P, no profiling, staging
    // size decided) the step is replayed from a CUDA graph captured once per
    // (particle buffer, key buffer) state; the launch sequence and its
    // arguments only depend on it.
    mpm_status stepOnce() {
        if (!steadyNow()) return stepBody();
        GraphSlot& g = graphs_[parity_][kcur_];
        const int p0 = parity_, k0 = kcur_;
        if (!g.exec) {
            MPM_TRY(captureGraph(g));
            if (!g.exec) return stepBody();
        }
        CUDA_TRY(cudaGraphLaunch(g.exec, stream_));
        noteLaunches(g.launches);
        advanceReplayed(p0, k0);
        return MPM_OK;
    }

    mpm_status stepBody() {
        if (!sorted_valid_) {
            MPM_TRY(sortLive());
        } else {
            // reusing the sort of initialize(): its mass pass counted nodes
            CUDA_TRY(cudaMemsetAsync(counters_.as<uint32_t>() + 2, 0, sizeof(uint32_t), stream_));
        }
        MPM_TRY(refreshStress());
        if (any_cfl_) launchCfl(ctx(), parity_, max_n_, err_.as<uint32_t>());
        graph_sorted_[parity_][kcur_] = sorted_;
        const int next = 1 - sorted_;
        StepArgs a = args(keys_[sorted_].as<uint32_t>(), vals_[sorted_].as<uint32_t>(), keys_[next].as<uint32_t>());
        LaunchCtx c = ctx();
        auto cs = combos();
        if (cs.size() > 1 && !profiling_ && !any_implicit_ && !tune_run_) {
            // Scenes of different (stencil, transfer) combinations share no
            // items, tiles or nodes: their P2G -> grid -> G2P chains run
            // concurrently, combination k on side stream k - 1, each with its
            // own work-item schedulers; the step joins them on the main stream.
            // (The autotuner times the combinations one after another: timed
            // side by side, its G2P choices for the 64-scene batch were worse.)
            MPM_TRY(ensureSideStreams((int)cs.size() - 1));
            CUDA_TRY(cudaEventRecord(fork_, stream_));
            for (size_t k = 0; k < cs.size(); ++k) {
                LaunchCtx ck = c;
                StepArgs ak = a;
                ak.sched = counters_.as<uint32_t>() + 8 + 8 * k;
                ak.spans = spans_.as<unsigned long long>() + (size_t)kSpanWords * k;
                if (k > 0) {
                    ck.stream = side_[k - 1];
                    CUDA_TRY(cudaStreamWaitEvent(ck.stream, fork_, 0));
                }
                const int mode = cs[k].transfer == MPM_TRANSFER_APIC ? MODE_APIC_FUSED : MODE_FLIP;
                ck.p2g_stage = p2gStageOf(cs[k]);
                ak.combo = (int)k;
                ak.p2g_lists = p2g_lists_.as<uint32_t>();
                ak.p2g_warp = warpModeOf(cs[k], k);
                launchP2G(ck, ak, cs[k].S, mode, cs[k].transfer);
                if (ak.p2g_warp != P2G_WARP_NONE) launchP2GWarp(ck, ak, cs[k].S, mode);
                launchGrid(ck, ak, cs[k].S, mode, cs[k].transfer);
                launchG2P(ck, ak, cs[k].S, cs[k].transfer == MPM_TRANSFER_APIC, true, (int)k);
                if (k > 0) {
                    CUDA_TRY(cudaEventRecord(join_[k - 1], ck.stream));
                    CUDA_TRY(cudaStreamWaitEvent(stream_, join_[k - 1], 0));
                }
            }
        } else {
            mark(KF_P2G, 0);
            for (size_t k = 0; k < cs.size(); ++k) {
                LaunchCtx ck = c;
                ck.p2g_stage = p2gStageOf(cs[k]);
                StepArgs ak = a;
                ak.spans = spans_.as<unsigned long long>() + (size_t)kSpanWords * k;
                if (tune_run_) CUDA_TRY(cudaEventRecord(tune_ev_[k][0], stream_));
                const int mode = cs[k].transfer == MPM_TRANSFER_APIC ? MODE_APIC_FUSED : MODE_FLIP;
                ak.combo = (int)k;
                ak.p2g_lists = p2g_lists_.as<uint32_t>();
                ak.p2g_warp = warpModeOf(cs[k], k);
                launchP2G(ck, ak, cs[k].S, mode, cs[k].transfer);
                if (ak.p2g_warp != P2G_WARP_NONE) launchP2GWarp(ck, ak, cs[k].S, mode);
                if (tune_run_) CUDA_TRY(cudaEventRecord(tune_ev_[k][1], stream_));
            }
            mark(KF_P2G, 1);
            collect(KF_P2G);
            mark(KF_GRID, 0);
            for (size_t k = 0; k < cs.size(); ++k) {
                StepArgs ak = a;
                ak.spans = spans_.as<unsigned long long>() + (size_t)kSpanWords * k;
                launchGrid(c, ak, cs[k].S, cs[k].transfer == MPM_TRANSFER_APIC ? MODE_APIC_FUSED : MODE_FLIP,
                           cs[k].transfer);
            }
            if (any_implicit_) MPM_TRY(launchSolveAll(false));
            mark(KF_GRID, 1);
            collect(KF_GRID);
            mark(KF_G2P, 0);
            for (size_t k = 0; k < cs.size(); ++k) {
                StepArgs ak = a;
                ak.spans = spans_.as<unsigned long long>() + (size_t)kSpanWords * k;
                if (tune_run_) CUDA_TRY(cudaEventRecord(tune_ev_[k][2], stream_));
                launchG2P(c, ak, cs[k].S, cs[k].transfer == MPM_TRANSFER_APIC, true, (int)k);
                if (tune_run_) CUDA_TRY(cudaEventRecord(tune_ev_[k][3], stream_));
            }
            mark(KF_G2P, 1);
            collect(KF_G2P);
        }
        CUDA_TRY(cudaGetLastError());
        parity_ ^= 1;
        kcur_ = next;
        keys_valid_ = true;   // G2P wrote next step's keys and block counts (and stress)
        sorted_valid_ = false;
        incremental_ok_ = true;  // the live order is now this step's sorted order
        return MPM_OK;
    }

    // ---- kernel spans measured on the device ------------------------------
    mpm_status resetSpans() {
        std::vector<unsigned long long> init((size_t)kSpanWords * kMaxCombos, 0ull);
        for (size_t i = 0; i < init.size(); i += 4) init[i] = ~0ull;
        CUDA_TRY(cudaMemcpyAsync(spans_.p, init.data(), init.size() * sizeof(unsigned long long),
                                 cudaMemcpyHostToDevice, stream_));
        CUDA_TRY(cudaStreamSynchronize(stream_));  // the host table is freed on return
        return MPM_OK;
    }
    // Per family (P2G, grid, G2P): the device time of the family's launches
    // per step (summed over the stencil/transfer combinations) and the number
    // of steps, since the last read; the counters restart.
    mpm_status readSpans(float* ms, int32_t* counts, int n) {
        if (!spans_.p) {
            for (int f = 0; f < n; ++f) {
                if (ms) ms[f] = 0.f;
                if (counts) counts[f] = 0;
            }
            return MPM_OK;
        }
        std::vector<unsigned long long> v((size_t)kSpanWords * kMaxCombos);
        CUDA_TRY(cudaStreamSynchronize(stream_));
        CUDA_TRY(cudaMemcpy(v.data(), spans_.p, v.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        for (int f = 0; f < n && f < SPAN_FAMILIES; ++f) {
            unsigned long long sum = 0, cnt = 0;
            for (int k = 0; k < kMaxCombos; ++k) {
                sum += v[(size_t)kSpanWords * k + 4 * f + 1];
                cnt = std::max(cnt, v[(size_t)kSpanWords * k + 4 * f + 2]);
            }
            if (ms) ms[f] = cnt ? (float)((double)sum / (double)cnt * 1e-6) : 0.f;
            if (counts) counts[f] = (int32_t)cnt;
        }
        return resetSpans();
    }

    // ---- launch settings and the autotuner ---------------------------------
    mpm_tuning tuningOf(int S, int transfer) const {
        auto it = tuning_.find({S, transfer});
        return it != tuning_.end() ? it->second : mpm_tuning{(int32_t)kDefaultG2PChunk, 0, -1};
    }
    // The P2G items of at most this many particles make combination c's
    // small list (list 0): its tuned warp threshold, or kWarpAutoMax.
    uint32_t warpMaxOf(const Combo& c) const {
        const int w = tuningOf(c.S, c.transfer).p2g_warp_max;
        return w >= 0 ? (uint32_t)w : kWarpAutoMax;
    }
    // Who takes the small list of combination k (index in combos()) this
    // step: with the engine's own choice (-1) the device decides from the
    // list's length (P2G_WARP_AUTO), unless the last read-back found too few
    // small items to launch the warp kernel at all.
    int warpModeOf(const Combo& c, size_t k) const {
        const int w = tuningOf(c.S, c.transfer).p2g_warp_max;
        if (w > 0) return P2G_WARP_ALWAYS;
        if (w == 0) return P2G_WARP_NONE;
        return (k < (size_t)kMaxCombos && !warp_few_[k]) ? P2G_WARP_AUTO : P2G_WARP_NONE;
    }
    int p2gStageOf(const Combo& c) const {
        const int st = tuningOf(c.S, c.transfer).p2g_stage;
        return st ? st : p2g_stage_;
    }
    ComboSplit comboSplit() const {
        ComboSplit g;
        for (int k = 0; k < kMaxCombos; ++k) {
            g.g2p_chunk[k] = kDefaultG2PChunk;
            g.p2g_warp_max[k] = 0;
        }
        auto cs = combos();
        for (size_t k = 0; k < cs.size() && k < (size_t)kMaxCombos; ++k) {
            g.g2p_chunk[k] = (uint32_t)tuningOf(cs[k].S, cs[k].transfer).g2p_chunk;
            g.p2g_warp_max[k] = warpMaxOf(cs[k]);
        }
        return g;
    }
    static mpm_status validTuning(const mpm_tuning& t) {
        if (t.g2p_chunk < (int)kMinG2PChunk || t.g2p_chunk > (int)kMaxG2PChunk)
            return fail(MPM_ERR_INVALID_ARG, "g2p_chunk must be in [MPM_G2P_CHUNK_MIN, MPM_G2P_CHUNK_MAX]");
        if (t.p2g_stage != 0 && t.p2g_stage != 16 && t.p2g_stage != 24 && t.p2g_stage != 32)
            return fail(MPM_ERR_INVALID_ARG, "p2g_stage must be 0, 16, 24 or 32");
        if (t.p2g_warp_max < -1 || t.p2g_warp_max > MPM_P2G_WARP_MAX_MAX)
            return fail(MPM_ERR_INVALID_ARG, "p2g_warp_max must be in [-1, MPM_P2G_WARP_MAX_MAX]");
        return MPM_OK;
    }
    // interpolation / transfer of -1 select every value.
    mpm_status setTuning(int interp, int transfer, const mpm_tuning& t) {
        MPM_TRY(validTuning(t));
        if (interp < -1 || interp > MPM_INTERP_CUBIC_BSPLINE || transfer < -1 || transfer > MPM_TRANSFER_APIC)
            return fail(MPM_ERR_INVALID_ARG, "unknown interpolation or transfer");
        CUDA_TRY(cudaStreamSynchronize(stream_));  // graphs in flight keep their settings
        for (int i = 0; i <= MPM_INTERP_CUBIC_BSPLINE; ++i)
            for (int tr = 0; tr <= MPM_TRANSFER_APIC; ++tr)
                if ((interp < 0 || interp == i) && (transfer < 0 || transfer == tr))
                    tuning_[{stencilSize(i), tr}] = t;
        dropGraphs();  // the captured launches carry the settings
        return MPM_OK;
    }
    mpm_status getTuning(int interp, int transfer, mpm_tuning* out) const {
        if (!out) return fail(MPM_ERR_INVALID_ARG, "null output");
        if (interp < 0 || interp > MPM_INTERP_CUBIC_BSPLINE || transfer < 0 || transfer > MPM_TRANSFER_APIC)
            return fail(MPM_ERR_INVALID_ARG, "unknown interpolation or transfer");
        *out = tuningOf(stencilSize(interp), transfer);
        return MPM_OK;
    }

    static int ppcBucket(double ppc) { return ppc < 2.0 ? 0 : ppc < 8.0 ? 1 : ppc < 32.0 ? 2 : 3; }

    // Times one round of candidate settings: one untimed step, then `steps`
    // steps with events around each combination's P2G and G2P launches;
    // adds the per-combination times (ms) to p2g_ms / g2p_ms.
    mpm_status tuneRound(int steps, std::vector<double>* p2g_ms, std::vector<double>* g2p_ms, int* run) {
        MPM_TRY(stepBody());
        advanceClock();
        ++*run;
        for (int i = 0; i < steps; ++i) {
            MPM_TRY(stepBody());
            advanceClock();
            ++*run;
            CUDA_TRY(cudaStreamSynchronize(stream_));
            for (size_t k = 0; k < tune_ev_.size(); ++k) {
                float a = 0.f, b = 0.f;
                CUDA_TRY(cudaEventElapsedTime(&a, tune_ev_[k][0], tune_ev_[k][1]));
                CUDA_TRY(cudaEventElapsedTime(&b, tune_ev_[k][2], tune_ev_[k][3]));
                (*p2g_ms)[k] += a;
                (*g2p_ms)[k] += b;
            }
        }
        return MPM_OK;
    }

    mpm_status autotune(int steps, int flags, int* steps_run) {
        int run = 0;
        if (steps_run) *steps_run = 0;
        if (steps < 1) return fail(MPM_ERR_INVALID_ARG, "steps_per_candidate must be >= 1");
        MPM_TRY(ensureReady());
        auto cs = combos();
        const size_t nc = cs.size();
        // device name (spaces replaced) for the cache key
        cudaDeviceProp prop{};
        CUDA_TRY(cudaGetDeviceProperties(&prop, device_));
        std::string dev = prop.name;
        for (auto& ch : dev)
            if (ch == ' ') ch = '_';
        std::map<std::pair<int, int>, mpm_tuning> saved = tuning_;
        for (size_t k = 0; k < nc; ++k) tuning_[{cs[k].S, cs[k].transfer}] = mpm_tuning{(int32_t)kMaxG2PChunk, 0, -1};
        dropGraphs();
        while (tune_ev_.size() < nc) {
            std::array<cudaEvent_t, 4> e4{};
            for (auto& e : e4) CUDA_TRY(cudaEventCreate(&e));
            tune_ev_.push_back(e4);
        }
        tune_run_ = true;
        struct Restore {
            Engine* e;
            ~Restore() {
                e->tune_run_ = false;
                e->dropGraphs();
            }
        } restore{this};
        // Key step: with one G2P item per block (chunk 4096) the G2P item
        // counts are the occupied blocks of each combination.
        MPM_TRY(stepBody());
        advanceClock();
        ++run;
        CUDA_TRY(cudaStreamSynchronize(stream_));
        if (stage_pending_) MPM_TRY(checkP2GStage());
        uint32_t cnt[kMaxCombos] = {};
        CUDA_TRY(cudaMemcpy(cnt, counters_.as<uint32_t>() + kG2PCountWord, sizeof(cnt), cudaMemcpyDeviceToHost));
        std::vector<std::string> keys(nc);
        std::vector<bool> todo(nc, false);
        bool any = false;
        {
            std::lock_guard<std::mutex> lock(g_tune_cache.mu);
            if (!(flags & MPM_TUNE_NO_DISK)) g_tune_cache.load();
            for (size_t k = 0; k < nc; ++k) {
                size_t n = 0;
                for (auto& sc : scenes_)
                    if (sc->S == cs[k].S && sc->desc.transfer == cs[k].transfer) n += sc->n;
                const double ppc = cnt[k] ? (double)n / (64.0 * cnt[k]) : 0.0;
                keys[k] = TuneCache::key(dev, cs[k].S, cs[k].transfer, ppcBucket(ppc));
                auto it = g_tune_cache.entries.find(keys[k]);
                if (it != g_tune_cache.entries.end() && !(flags & MPM_TUNE_FORCE)) {
                    saved[{cs[k].S, cs[k].transfer}] = it->second;
                } else {
                    todo[k] = true;
                    any = true;
                }
            }
        }
        if (any) {
            // round r: G2P chunk r, P2G staging size r mod 3 (the two kernels
            // do not depend on each other's setting).  The P2G warp threshold
            // stays the engine's choice (-1): searched per combination over a
            // few steps it chose worse than the item-count rule (64-scene
            // batch 1.92-1.96 ms against 1.87).
            const uint32_t chunks[] = {256, 512, 1024, 2048, 4096};
            const int stages[] = {16, 24, 32};
            std::vector<double> best_g2p(nc, 1e30), p2g_sum[3], p2g_cnt(3, 0.0);
            std::vector<uint32_t> best_chunk(nc, kDefaultG2PChunk);
            for (auto& v : p2g_sum) v.assign(nc, 0.0);
            for (int r = 0; r < 5; ++r) {
                const int st = r % 3;
                for (size_t k = 0; k < nc; ++k)
                    if (todo[k]) tuning_[{cs[k].S, cs[k].transfer}] = mpm_tuning{(int32_t)chunks[r], stages[st], -1};
                std::vector<double> pm(nc, 0.0), gm(nc, 0.0);
                MPM_TRY(tuneRound(steps, &pm, &gm, &run));
                for (size_t k = 0; k < nc; ++k) {
                    if (gm[k] < best_g2p[k]) {
                        best_g2p[k] = gm[k];
                        best_chunk[k] = chunks[r];
                    }
                    p2g_sum[st][k] += pm[k];
                }
                p2g_cnt[st] += 1.0;
            }
            std::lock_guard<std::mutex> lock(g_tune_cache.mu);
            for (size_t k = 0; k < nc; ++k) {
                if (!todo[k]) continue;
                int bs = 32;
                double bt = 1e30;
                for (int st = 0; st < 3; ++st) {
                    const double t = p2g_sum[st][k] / p2g_cnt[st];
                    if (t < bt) {
                        bt = t;
                        bs = stages[st];
                    }
                }
                const mpm_tuning t{(int32_t)best_chunk[k], bs, -1};
                saved[{cs[k].S, cs[k].transfer}] = t;
                g_tune_cache.store(keys[k], t, !(flags & MPM_TUNE_NO_DISK));
            }
        }
        tuning_ = saved;
        if (steps_run) *steps_run = run;
        return MPM_OK;
    }

    // P2G stages 32 particles per warp pass in dense scenes and 16 in sparse
    // ones (fewer than 8 particles per cell on average: the smaller staging
    // buffer fits 3 CTAs per SM and the passes are rarely full).  Decided
    // once after the first step that follows a change of the scene set,
    // from the number of work items of that step.  The count is read back
    // asynchronously (a copy into pinned host memory and an event), so the
    // host does not wait for the GPU: the steps that follow run with direct
    // launches until the event has completed, and only then is the step
    // captured as a CUDA graph (a change of staging size would drop it).
    mpm_status checkP2GStage() {
        if (!stage_check_) return MPM_OK;
        if (!stage_pending_) {
            if (!host_word_) {
                host_word_ = g_pinned_words.take();
                if (!host_word_) return fail(MPM_ERR_OOM, "no page-locked host word for the staging read-back");
                CUDA_TRY(cudaEventCreateWithFlags(&stage_event_, cudaEventDisableTiming));
            }
            CUDA_TRY(cudaMemcpyAsync(host_word_, counters_.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_));
            static_assert(1 + kMaxCombos <= PinnedWords::kLine, "read-back line too short");
            CUDA_TRY(cudaMemcpyAsync(host_word_ + 1, counters_.as<uint32_t>() + kP2GSmallWord,
                                     sizeof(uint32_t) * kMaxCombos, cudaMemcpyDeviceToHost, stream_));
            CUDA_TRY(cudaEventRecord(stage_event_, stream_));
            stage_pending_ = true;
            return MPM_OK;
        }
        const cudaError_t q = cudaEventQuery(stage_event_);
        if (q == cudaErrorNotReady) return MPM_OK;
        CUDA_TRY(q);
        stage_pending_ = false;
        stage_check_ = false;
        const uint32_t items = host_word_[0];
        const int stage = (items > 0 && ntot_ / items < 512) ? 16 : 32;
        bool changed = stage != p2g_stage_;
        p2g_stage_ = stage;
        // a combination with too few small P2G items for warps skips the
        // warp kernel's launch (the device would leave them to p2gKernel)
        for (int k = 0; k < kMaxCombos; ++k) {
            const bool few = host_word_[1 + k] < kWarpAutoMinItems;
            changed |= few != warp_few_[k];
            warp_few_[k] = few;
        }
        if (changed) dropGraphs();
        return MPM_OK;
    }

    mpm_status step(int n) {
        if (n < 0) return fail(MPM_ERR_INVALID_ARG, "nsteps must be >= 0");
        MPM_TRY(ensureReady());
        for (int i = 0; i < n; ++i) {
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (step_timing_) {
                MPM_TRY(timingEvent(&e0));
                MPM_TRY(timingEvent(&e1));
                CUDA_TRY(cudaEventRecord(e0, stream_));
            }
            MPM_TRY(stepOnce());
            if (step_timing_) {
                CUDA_TRY(cudaEventRecord(e1, stream_));
                step_events_.push_back({e0, e1});
            }
            MPM_TRY(checkP2GStage());
            advanceClock();
        }
        return MPM_OK;
    }

    // ---- per-step device times without host synchronization ---------------
    // With step timing on, every step is bracketed by two events on the
    // stream; stepTimes() hands out the device times of the steps that have
    // completed (oldest first) without waiting, waitSteps() blocks until at
    // most `in_flight` timed steps are still queued or running.
    mpm_status timingEvent(cudaEvent_t* e) {
        if (!free_events_.empty()) {
            *e = free_events_.back();
            free_events_.pop_back();
            return MPM_OK;
        }
        CUDA_TRY(cudaEventCreate(e));
        return MPM_OK;
    }
    mpm_status setStepTiming(bool on) {
        step_timing_ = on;
        if (!on) {
            CUDA_TRY(cudaStreamSynchronize(stream_));
            for (auto& p : step_events_) {
                free_events_.push_back(p.first);
                free_events_.push_back(p.second);
            }
            step_events_.clear();
        }
        return MPM_OK;
    }
    mpm_status stepTimes(float* ms, int cap, int* count) {
        int k = 0;
        while (!step_events_.empty() && k < cap) {
            auto [e0, e1] = step_events_.front();
            const cudaError_t q = cudaEventQuery(e1);
            if (q == cudaErrorNotReady) break;
            CUDA_TRY(q);
            float t = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
            if (ms) ms[k] = t;
            ++k;
            step_events_.pop_front();
            free_events_.push_back(e0);
            free_events_.push_back(e1);
        }
        if (count) *count = k;
        return MPM_OK;
    }
    mpm_status waitSteps(int in_flight) {
        if (in_flight < 0) return fail(MPM_ERR_INVALID_ARG, "in_flight must be >= 0");
        const int n = (int)step_events_.size();
        if (n > in_flight) CUDA_TRY(cudaEventSynchronize(step_events_[n - 1 - in_flight].second));
        return MPM_OK;
    }

    void advanceClock() {
        for (auto& s : scenes_) {
            s->last_cfl = s->cfl > 0.f;
            if (!s->last_cfl) {
                s->time_fixed += (double)s->desc.dt;
                s->last_dt = s->desc.dt;
            }
        }
    }

    // CFL time step of a scene: cfl > 0 makes every step's dt
    // min(desc.dt, cfl h / max_p |v_p|) from the velocities the step starts
    // with; 0 returns to the fixed desc.dt.
    mpm_status setCfl(int id, float cfl) {
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        if (!(cfl >= 0.f) || !std::isfinite(cfl)) return fail(MPM_ERR_INVALID_ARG, "cfl must be finite and >= 0");
        scenes_[idx]->cfl = cfl;
        if (!dirty_) {
            host_scenes_[idx].cfl = cfl;
            MPM_TRY(uploadSceneTable());
        }
        bool any = false;
        for (auto& s : scenes_) any |= s->cfl > 0.f;
        if (any != any_cfl_) {  // the step's launch sequence changes
            CUDA_TRY(cudaStreamSynchronize(stream_));
            any_cfl_ = any;
            dropGraphs();
        }
        return MPM_OK;
    }

    // Simulated time advanced by step() and the dt of the last step.
    mpm_status simTime(int id, double* t, float* last_dt) {
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        SceneHost& s = *scenes_[idx];
        CflState st{};
        CUDA_TRY(cudaStreamSynchronize(stream_));
        CUDA_TRY(cudaMemcpy(&st, s.cfl_state.p, sizeof(CflState), cudaMemcpyDeviceToHost));
        if (t) *t = s.time_fixed + st.time;
        if (last_dt) *last_dt = s.last_cfl ? st.last_dt : s.last_dt;
        return MPM_OK;
    }

    mpm_status timedStep(int n, float* ms) {
        if (!ms) return fail(MPM_ERR_INVALID_ARG, "null output");
        MPM_TRY(ensureReady());
        MPM_TRY(prepareGraphs());
        CUDA_TRY(cudaEventRecord(ev_[0][0], stream_));
        for (int i = 0; i < n; ++i) {
            MPM_TRY(stepOnce());
            MPM_TRY(checkP2GStage());
            advanceClock();
        }
        CUDA_TRY(cudaEventRecord(ev_[0][1], stream_));
        CUDA_TRY(cudaEventSynchronize(ev_[0][1]));
        CUDA_TRY(cudaEventElapsedTime(ms, ev_[0][0], ev_[0][1]));
        return MPM_OK;
    }

    mpm_status accumulateProfile() {
        if (records_.empty()) return MPM_OK;
        CUDA_TRY(cudaStreamSynchronize(stream_));
        for (auto& r : records_) {
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, r.e0, r.e1));
            prof_ms_[r.fam] += ms;
            prof_cnt_[r.fam] += 1;
            event_pool_.push_back(r.e0);
            event_pool_.push_back(r.e1);
        }
        records_.clear();
        return MPM_OK;
    }

    mpm_status stats(mpm_step_stats* out) {
        if (!out) return fail(MPM_ERR_INVALID_ARG, "null output");
        *out = mpm_step_stats{};
        if (dirty_ || !counters_.p) return MPM_OK;
        uint32_t c[4] = {0, 0, 0, 0};
        CUDA_TRY(cudaStreamSynchronize(stream_));
        CUDA_TRY(cudaMemcpy(c, counters_.p, sizeof(c), cudaMemcpyDeviceToHost));
        out->active_blocks = c[0];
        out->outside_blocks = c[1];
        out->active_nodes = c[2];
        return MPM_OK;
    }

    mpm_status synchronize() {
        CUDA_TRY(cudaStreamSynchronize(stream_));
        if (stage_pending_) MPM_TRY(checkP2GStage());  // its read-back has landed
        MPM_TRY(downloadWait());
        uint32_t e = 0;
        CUDA_TRY(cudaMemcpy(&e, err_.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (e) {
            CUDA_TRY(cudaMemset(err_.p, 0, sizeof(uint32_t)));
            if (e & ERR_NONFINITE) return fail(MPM_ERR_NUMERIC, "non-finite particle position detected on the device");
            if (e & ERR_WAIT_TIMEOUT)
                return fail(MPM_ERR_TIMEOUT, "a bounded wait for a G2P grid tile gave up; recreate the solver");
            return fail(MPM_ERR_CUDA, "device error flag " + std::to_string(e));
        }
        return MPM_OK;
    }

    // ---- split API --------------------------------------------------------
    mpm_status ensureDbg() {
        bool changed = false;
        for (auto& s : scenes_)
            if (!s->dbg.p) {
                MPM_TRY(alloc(s->dbg, sizeof(float) * 10 * s->nodes(), "dense debug grid"));
                CUDA_TRY(cudaMemsetAsync(s->dbg.p, 0, sizeof(float) * 10 * s->nodes(), stream_));
                changed = true;
            }
        if (changed) {
            for (size_t i = 0; i < scenes_.size(); ++i) host_scenes_[i].dbg = scenes_[i]->dbg.as<float>();
            MPM_TRY(uploadSceneTable());
        }
        return MPM_OK;
    }
    mpm_status resetGrid() {
        MPM_TRY(ensureReady());
        MPM_TRY(ensureDbg());
        for (auto& s : scenes_) CUDA_TRY(cudaMemsetAsync(s->dbg.p, 0, sizeof(float) * 10 * s->nodes(), stream_));
        return MPM_OK;
    }
    mpm_status particlesToGrid() {
        MPM_TRY(ensureReady());
        MPM_TRY(ensureDbg());
        MPM_TRY(sortLive());
        MPM_TRY(refreshStress());
        StepArgs a = args(keys_[sorted_].as<uint32_t>(), vals_[sorted_].as<uint32_t>(), nullptr);
        LaunchCtx c = ctx();
        for (int S : stencilSizes()) {
            launchP2G(c, a, S, MODE_SPLIT, -1);
            launchGrid(c, a, S, MODE_SPLIT, -1);
        }
        CUDA_TRY(cudaGetLastError());
        keys_valid_ = false;
        return MPM_OK;
    }
    mpm_status gravity() {
        MPM_TRY(ensureReady());
        MPM_TRY(ensureDbg());
        launchDenseGravity(ctx());
        CUDA_TRY(cudaGetLastError());
        return MPM_OK;
    }
    mpm_status updateGridVelocities(float dt) {
        MPM_TRY(ensureReady());
        MPM_TRY(ensureDbg());
        launchDenseUpdate(ctx(), dt);
        CUDA_TRY(cudaGetLastError());
        return MPM_OK;
    }
    mpm_status gridCollision(float dt) {
        MPM_TRY(ensureReady());
        MPM_TRY(ensureDbg());
        launchDenseCollision(ctx(), dt);
        CUDA_TRY(cudaGetLastError());
        return MPM_OK;
    }
    mpm_status gridToParticles(float dt, float blend, bool override_blend) {
        MPM_TRY(ensureReady());
        MPM_TRY(ensureDbg());
        if (!sorted_valid_) MPM_TRY(sortLive());
        MPM_TRY(refreshStress());
        launchDensePack(ctx());
        std::vector<SceneDev> saved = host_scenes_;
        for (auto& d : host_scenes_) {
            d.dt = dt;
            if (override_blend) d.blend = blend;
        }
        MPM_TRY(uploadSceneTable());
        StepArgs a = args(keys_[sorted_].as<uint32_t>(), vals_[sorted_].as<uint32_t>(), nullptr);
        LaunchCtx c = ctx();
        {
            auto cs = combos();
            for (size_t k = 0; k < cs.size(); ++k)
                launchG2P(c, a, cs[k].S, cs[k].transfer == MPM_TRANSFER_APIC, false, (int)k);
        }
        CUDA_TRY(cudaGetLastError());
        host_scenes_ = saved;
        MPM_TRY(uploadSceneTable());
        parity_ ^= 1;
        keys_valid_ = false;
        sorted_valid_ = false;
        return MPM_OK;
    }
    mpm_status particlesCollision(float dt) {
        MPM_TRY(ensureReady());
        launchParticlesCollision(ctx(), parity_, dt);
        CUDA_TRY(cudaGetLastError());
        return MPM_OK;
    }
    mpm_status advect(float dt) {
        MPM_TRY(ensureReady());
        launchAdvect(ctx(), parity_, dt);
        CUDA_TRY(cudaGetLastError());
        keys_valid_ = false;
        sorted_valid_ = false;
        return MPM_OK;
    }

    // ---- data movement ----------------------------------------------------
    static int fieldInfo(int field, int* base, int* comps, int* mode) {
        *mode = 0;
        switch (field) {
            case MPM_FIELD_POSITION: *base = F_X; *comps = 3; return 3;
            case MPM_FIELD_VELOCITY: *base = F_V; *comps = 3; return 3;
            case MPM_FIELD_FE: *base = F_FE; *comps = 9; return 9;
            case MPM_FIELD_FP: *base = F_FP; *comps = 9; return 9;
            case MPM_FIELD_B: *base = F_B; *comps = 9; return 9;
            case MPM_FIELD_VOLUME0: *base = F_VOL; *comps = 1; return 1;
            case MPM_FIELD_MASS: *base = F_MASS; *comps = 1; return 1;
            case MPM_FIELD_POSITION4: *base = F_X; *comps = 4; *mode = 1; return 4;
            case MPM_FIELD_DET_FE: *base = F_FE; *comps = 1; *mode = 2; return 1;
            case MPM_FIELD_DET_FP: *base = F_FP; *comps = 1; *mode = 2; return 1;
            default: return 0;
        }
    }

    mpm_status download(int id, int field, float* host, bool sync = true) {
        MPM_TRY(ensureReady());
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        if (!host) return fail(MPM_ERR_INVALID_ARG, "null output pointer");
        int base, comps, mode;
        int per = fieldInfo(field, &base, &comps, &mode);
        if (!per) return fail(MPM_ERR_INVALID_ARG, "unknown particle field");
        SceneHost& s = *scenes_[idx];
        if (field == MPM_FIELD_B && s.desc.transfer != MPM_TRANSFER_APIC)
            return fail(MPM_ERR_INVALID_ARG, "B is only defined for APIC scenes");
        if (s.n == 0) return MPM_OK;
        const size_t bytes = sizeof(float) * per * s.n;
        MPM_TRY(alloc(tmp_, bytes, "download buffer"));
        LaunchCtx c = ctx();
        launchGatherField(c, idx, parity_, base, comps, mode, tmp_.as<float>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(host, tmp_.p, bytes, cudaMemcpyDeviceToHost, stream_));
        if (sync) return synchronize();
        return MPM_OK;
    }

    // Asynchronous download: the gather into one of the scene's two device
    // staging buffers runs in stream order (it reads the current state), the
    // copy to the host runs on a separate copy stream, so it overlaps the
    // steps that follow (they write the other particle buffer and never the
    // staging buffers).  A staging buffer is reused only after its previous
    // copy has finished (the compute stream waits for that copy's event).
    mpm_status downloadAsync(int id, int field, float* host) {
        MPM_TRY(ensureReady());
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        if (!host) return fail(MPM_ERR_INVALID_ARG, "null output pointer");
        int base, comps, mode;
        int per = fieldInfo(field, &base, &comps, &mode);
        if (!per) return fail(MPM_ERR_INVALID_ARG, "unknown particle field");
        SceneHost& s = *scenes_[idx];
        if (field == MPM_FIELD_B && s.desc.transfer != MPM_TRANSFER_APIC)
            return fail(MPM_ERR_INVALID_ARG, "B is only defined for APIC scenes");
        if (s.n == 0) return MPM_OK;
        if (!copy_stream_) CUDA_TRY(takeStream(device_, &copy_stream_));
        if (!s.stage_ready[0])
            for (int k = 0; k < 2; ++k) {
                CUDA_TRY(cudaEventCreateWithFlags(&s.stage_ready[k], cudaEventDisableTiming));
                CUDA_TRY(cudaEventCreateWithFlags(&s.stage_done[k], cudaEventDisableTiming));
            }
        const int k = s.stage_next;
        s.stage_next ^= 1;
        const size_t bytes = sizeof(float) * per * s.n;
        if (s.stage[k].bytes < bytes) {
            if (s.stage_pending[k]) CUDA_TRY(cudaEventSynchronize(s.stage_done[k]));
            mpm_status pst;
            cudaMemPool_t pool = scenePool(device_, &pst);
            if (!pool) return pst;
            MPM_TRY(s.stage[k].allocPooled(bytes, "download staging buffer", pool, stream_));
        }
        if (s.stage_pending[k]) CUDA_TRY(cudaStreamWaitEvent(stream_, s.stage_done[k], 0));
        launchGatherField(ctx(), idx, parity_, base, comps, mode, s.stage[k].as<float>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaEventRecord(s.stage_ready[k], stream_));
        CUDA_TRY(cudaStreamWaitEvent(copy_stream_, s.stage_ready[k], 0));
        CUDA_TRY(cudaMemcpyAsync(host, s.stage[k].p, bytes, cudaMemcpyDeviceToHost, copy_stream_));
        CUDA_TRY(cudaEventRecord(s.stage_done[k], copy_stream_));
        s.stage_pending[k] = true;
        return MPM_OK;
    }

    // Waits for every asynchronous download issued so far.
    mpm_status downloadWait() {
        if (!copy_stream_) return MPM_OK;
        CUDA_TRY(cudaStreamSynchronize(copy_stream_));
        for (auto& s : scenes_) s->stage_pending[0] = s->stage_pending[1] = false;
        return MPM_OK;
    }

    // Density of one scene on its dense grid (res^3 floats, node index
    // x + X (y + Y z)): a mass pass of that scene alone on a cleared grid, then
    // m / h^3 per node.  The particle state is not changed: the next step
    // continues exactly as without this call.
    mpm_status downloadDensity(int id, float* host) {
        MPM_TRY(ensureReady());
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        if (!host) return fail(MPM_ERR_INVALID_ARG, "null output pointer");
        SceneHost& s = *scenes_[idx];
        const size_t nodes = s.nodes();
        CUDA_TRY(cudaMemsetAsync(s.vstar.p, 0, sizeof(float4) * nodes, stream_));
        if (s.n > 0) {
            for (size_t i = 0; i < scenes_.size(); ++i) host_scenes_[i].init_pass = (int)(i == (size_t)idx);
            MPM_TRY(uploadSceneTable());
            if (!sorted_valid_) MPM_TRY(sortLive());
            StepArgs a = args(keys_[sorted_].as<uint32_t>(), vals_[sorted_].as<uint32_t>(), nullptr);
            LaunchCtx c = ctx();
            launchP2G(c, a, s.S, MODE_MASS, -1);
            launchGrid(c, a, s.S, MODE_MASS, -1);
            keys_valid_ = false;  // block counts were consumed by the compaction
        }
        // cell_vol_inv as the reference forms it: 1.0 / (h*h*h) in double, stored as float
        const float h = s.desc.stride;
        const float inv = (float)(1.0 / (double)(h * h * h));
        MPM_TRY(grow(tmp_, sizeof(float) * nodes, "density buffer"));
        launchDensity(ctx(), s.vstar.as<float4>(), nodes, inv, tmp_.as<float>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemcpyAsync(host, tmp_.p, sizeof(float) * nodes, cudaMemcpyDeviceToHost, stream_));
        return synchronize();
    }

    mpm_status upload(int id, int field, const float* host) {
        MPM_TRY(ensureReady());
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        if (!host) return fail(MPM_ERR_INVALID_ARG, "null input pointer");
        int base, comps, mode;
        int per = fieldInfo(field, &base, &comps, &mode);
        if (!per || mode != 0 || field == MPM_FIELD_MASS)
            return fail(MPM_ERR_INVALID_ARG, "field cannot be uploaded");
        SceneHost& s = *scenes_[idx];
        if (s.n == 0) return MPM_OK;
        const size_t bytes = sizeof(float) * per * s.n;
        MPM_TRY(alloc(tmp_, bytes, "upload buffer"));
        CUDA_TRY(cudaMemcpyAsync(tmp_.p, host, bytes, cudaMemcpyHostToDevice, stream_));
        launchScatterField(ctx(), idx, parity_, base, comps, tmp_.as<float>());
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamSynchronize(stream_));
        s.stress_stale = true;
        if (field == MPM_FIELD_POSITION) {
            keys_valid_ = false;
            sorted_valid_ = false;
        }
        return MPM_OK;
    }

    mpm_status downloadGrid(int id, int field, float* host) {
        MPM_TRY(ensureReady());
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        SceneHost& s = *scenes_[idx];
        if (!s.dbg.p) return fail(MPM_ERR_INVALID_ARG, "the dense grid exists only after split-API grid calls");
        const size_t nodes = s.nodes();
        std::vector<float> planes;
        int first, comps;
        switch (field) {
            case MPM_GRID_MASS: first = 0; comps = 1; break;
            case MPM_GRID_VELOCITY: first = 1; comps = 3; break;
            case MPM_GRID_FORCE: first = 4; comps = 3; break;
            case MPM_GRID_VELOCITY_STAR: first = 7; comps = 3; break;
            default: return fail(MPM_ERR_INVALID_ARG, "unknown grid field");
        }
        planes.resize(nodes * comps);
        CUDA_TRY(cudaMemcpyAsync(planes.data(), s.dbg.as<float>() + first * nodes, sizeof(float) * nodes * comps,
                                 cudaMemcpyDeviceToHost, stream_));
        CUDA_TRY(cudaStreamSynchronize(stream_));
        for (size_t i = 0; i < nodes; ++i)
            for (int c = 0; c < comps; ++c) host[comps * i + c] = planes[c * nodes + i];
        return MPM_OK;
    }

    mpm_status setParticlesCollision(int id, int enable) {
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        scenes_[idx]->desc.particles_collision = enable ? 1 : 0;
        if (!dirty_) {
            host_scenes_[idx].pcoll = enable ? 1 : 0;
            MPM_TRY(uploadSceneTable());
        }
        return MPM_OK;
    }

    // Level-set collision object of a scene: phi holds the signed distance at
    // every grid node (index x + X(y + Y z), world units, negative inside),
    // or is null to remove the object.
    mpm_status setLevelSet(int id, const float* phi, float friction, const float* velocity) {
        int idx = sceneIndex(id);
        if (idx < 0) return fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        SceneHost& s = *scenes_[idx];
        if (phi) {
            for (int a = 0; a < 3; ++a)
                if (s.desc.resolution[a] < 2) return fail(MPM_ERR_INVALID_ARG, "a level set needs >= 2 nodes per axis");
            if (!(friction >= 0.f) || !std::isfinite(friction))
                return fail(MPM_ERR_INVALID_ARG, "level-set friction must be finite and >= 0");
            if (velocity)
                for (int a = 0; a < 3; ++a)
                    if (!std::isfinite(velocity[a])) return fail(MPM_ERR_INVALID_ARG, "level-set velocity not finite");
            const size_t nodes = s.nodes();
            for (size_t i = 0; i < nodes; ++i)
                if (!std::isfinite(phi[i])) return fail(MPM_ERR_INVALID_ARG, "level set has a non-finite value");
            CUDA_TRY(cudaStreamSynchronize(stream_));  // earlier steps may still read the old values
            MPM_TRY(grow(s.phi, sizeof(float) * nodes, "level set"));
            CUDA_TRY(cudaMemcpy(s.phi.p, phi, sizeof(float) * nodes, cudaMemcpyHostToDevice));
            s.has_phi = true;
            s.phi_friction = friction;
            for (int a = 0; a < 3; ++a) s.phi_vel[a] = velocity ? velocity[a] : 0.f;
        } else {
            s.has_phi = false;
        }
        if (!dirty_) {
            SceneDev& d = host_scenes_[idx];
            d.phi = s.has_phi ? s.phi.as<float>() : nullptr;
            d.phi_friction = s.phi_friction;
            for (int a = 0; a < 3; ++a) d.phi_vel[a] = s.phi_vel[a];
            MPM_TRY(uploadSceneTable());
        }
        return MPM_OK;
    }

    mpm_status profile(int enable) {
        MPM_TRY(accumulateProfile());
        if (enable) {
            for (int k = 0; k < KF_COUNT; ++k) {
                prof_ms_[k] = 0;
                prof_cnt_[k] = 0;
            }
        }
        profiling_ = enable != 0;
        return MPM_OK;
    }
    mpm_status profileRead(float* ms, int32_t* counts, int nf) {
        MPM_TRY(accumulateProfile());
        for (int k = 0; k < nf && k < KF_COUNT; ++k) {
            if (ms) ms[k] = prof_cnt_[k] ? (float)(prof_ms_[k] / prof_cnt_[k]) : 0.f;
            if (counts) counts[k] = prof_cnt_[k];
        }
        return MPM_OK;
    }

    size_t numScenes() const { return scenes_.size(); }
    size_t totalParticles() const {
        size_t n = 0;
        for (auto& s : scenes_) n += s->n;
        return n;
    }
    cudaStream_t stream() const { return stream_; }

private:
    int device_ = 0, num_sms_ = 148;
    cudaMemPool_t pool_ = nullptr;         // the device's scene pool (init)
    size_t staging_reserved_ = 0;          // particles whose download staging the pool was grown for
    uint32_t* host_word_ = nullptr;        // pinned: work-item count read back by checkP2GStage
    cudaEvent_t stage_event_ = nullptr;    // completion of that read-back
    bool stage_pending_ = false;
    cudaStream_t stream_ = nullptr;
    cudaStream_t compact_stream_ = nullptr;  // block compaction beside the sort
    cudaEvent_t compact_fork_ = nullptr, compact_join_ = nullptr;
    std::vector<std::unique_ptr<SceneHost>> scenes_;
    std::vector<SceneDev> host_scenes_;
    int next_id_ = 0;
    bool dirty_ = true, keys_valid_ = false, sorted_valid_ = false;
    bool any_cfl_ = false;     // some scene steps with a CFL dt (two more launches per step)
    bool any_implicit_ = false;  // some scene solves the semi-implicit update
    DevMem cell_range_, block_range_, solve_pofs_, solve_prep_, solve_T_, solve_iter_;
    int p2g_stage_ = 32;       // see checkP2GStage()
    uint32_t g2p_cap_ = 1;   // G2P items per combination (rebuild)
    // launch settings per (stencil, transfer) combination (mpm_tuning)
    std::map<std::pair<int, int>, mpm_tuning> tuning_;
    bool tune_run_ = false;                          // autotune: sequential launches with events
    std::vector<std::array<cudaEvent_t, 4>> tune_ev_;  // per combination: P2G start/end, G2P start/end
    bool stage_check_ = true;
    // the previous step's sorted keys are aligned with the live particle order
    // (sortLive may sort incrementally); MPM_FULL_SORT=1 always sorts all keys,
    // MPM_INCREMENTAL_SORT=1 sorts incrementally whatever the size (both for
    // tests and measurements)
    bool incremental_ok_ = false;
    const bool full_sort_only_ = getenv("MPM_FULL_SORT") != nullptr;
    const bool incremental_always_ = getenv("MPM_INCREMENTAL_SORT") != nullptr;
    // Below this many keys the full radix sort is faster (the movers' sort
    // costs a few fixed-latency passes): 1M keys 0.072 ms full vs 0.100 ms
    // incremental, 8.5M keys 0.43 ms vs 0.30 ms on the B200.
    static constexpr size_t kIncrementalMinKeys = (size_t)3 << 20;
    int parity_ = 0, kcur_ = 0, sorted_ = 0;
    size_t ntot_ = 0, max_nodes_ = 0, max_n_ = 0, max_active_ = 1, tile_stride_ = 0;
    uint32_t total_blocks_ = 0;
    int key_bits_ = 1;
    DevMem keys_[2], vals_[2], sort_scratch_, inc_scratch_, compact_scratch_, block_count_, sbb_, active_,
        outside_, counters_, block_slot_, tiles_, scenes_dev_, err_, tmp_, g2p_items_, tmaps_, spans_, p2g_lists_;
    // Per combination: the first step after a change of the scene set found
    // fewer than kWarpAutoMinItems small P2G items, so the step does not
    // launch the warp kernel (see checkP2GStage, warpModeOf).
    bool warp_few_[kMaxCombos] = {};
    bool profiling_ = false;
    bool step_timing_ = false;
    std::deque<std::pair<cudaEvent_t, cudaEvent_t>> step_events_;
    std::vector<cudaEvent_t> free_events_;
    cudaStream_t copy_stream_ = nullptr;  // asynchronous downloads (downloadAsync)
    // side streams of the concurrent per-combination chains (stepBody)
    static constexpr int kMaxSide = 5;
    cudaStream_t side_[kMaxSide] = {};
    cudaEvent_t fork_ = nullptr, join_[kMaxSide] = {};
    mpm_status ensureSideStreams(int n) {
        if (n > kMaxSide) return fail(MPM_ERR_UNSUPPORTED, "too many stencil/transfer combinations");
        if (!fork_) CUDA_TRY(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
        for (int k = 0; k < n; ++k)
            if (!side_[k]) {
                CUDA_TRY(takeStream(device_, &side_[k]));
                CUDA_TRY(cudaEventCreateWithFlags(&join_[k], cudaEventDisableTiming));
            }
        return MPM_OK;
    }
    GraphSlot graphs_[2][2];          // [particle buffer parity][unsorted key buffer]
    int graph_sorted_[2][2] = {};     // sorted key buffer after the sort of that state
    bool use_graphs_ = getenv("MPM_NO_GRAPHS") == nullptr;
    void dropGraphs() {
        for (auto& row : graphs_)
            for (auto& g : row) {
                if (g.exec) cudaGraphExecDestroy(g.exec);
                g.exec = nullptr;
            }
    }
    cudaEvent_t ev_[KF_COUNT][2] = {};
    struct Record {
        int fam;
        cudaEvent_t e0, e1;
    };
    std::vector<Record> records_;
    std::vector<cudaEvent_t> event_pool_;
    cudaEvent_t open_[KF_COUNT] = {};
    double prof_ms_[KF_COUNT] = {};
    int prof_cnt_[KF_COUNT] = {};
};

}  // namespace mpm

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using mpm::Engine;

struct mpm_solver {
    Engine eng;
    int scene = -1;
};

struct mpm_batch {
    Engine eng;
};

#define GUARD(expr)                                                     \
    try {                                                               \
        return (expr);                                                  \
    } catch (const std::bad_alloc&) {                                   \
        return mpm::fail(MPM_ERR_OOM, "host allocation failed");        \
    } catch (const std::exception& e) {                                 \
        return mpm::fail(MPM_ERR_CUDA, e.what());                       \
    }

extern "C" {

int32_t mpm_abi_version(void) { return MPM_B200_ABI_VERSION; }

const char* mpm_last_error_string(void) { return mpm::g_last_error.c_str(); }

mpm_status mpm_device_count(int32_t* count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        n = 0;
    }
    if (count) *count = n;
    return MPM_OK;
}

static mpm_status check(const mpm_solver* s) {
    if (!s) return mpm::fail(MPM_ERR_INVALID_ARG, "null solver handle");
    return MPM_OK;
}

mpm_status mpm_solver_create(const mpm_scene_desc* desc, const mpm_particles_in* particles, mpm_solver** out) {
    if (!desc || !particles || !out) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    try {
        mpm_status st = Engine::validate(*desc, *particles);
        if (st != MPM_OK) return st;
        std::unique_ptr<mpm_solver> s(new mpm_solver);
        st = s->eng.init();
        if (st != MPM_OK) return st;
        st = s->eng.addScene(*desc, *particles, &s->scene);
        if (st != MPM_OK) return st;
        st = s->eng.ensureReady();
        if (st != MPM_OK) return st;
        st = s->eng.synchronize();
        if (st != MPM_OK) return st;
        *out = s.release();
        return MPM_OK;
    } catch (const std::bad_alloc&) {
        return mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
}

mpm_status mpm_solver_destroy(mpm_solver* s) {
    if (!s) return MPM_OK;
    cudaStreamSynchronize(s->eng.stream());
    delete s;
    return MPM_OK;
}

mpm_status mpm_solver_save(mpm_solver* s, const char* path) {
    MPM_TRY(check(s));
    return s->eng.saveScene(s->scene, path);
}

mpm_status mpm_solver_load(const char* path, mpm_solver** out) {
    if (!out) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    try {
        Engine::Checkpoint ck;
        mpm_status st = Engine::readCheckpoint(path, &ck);  // host only: checked before any device work
        if (st != MPM_OK) return st;
        std::unique_ptr<mpm_solver> s(new mpm_solver);
        st = s->eng.init();
        if (st != MPM_OK) return st;
        st = s->eng.loadScene(ck, &s->scene);
        if (st != MPM_OK) return st;
        st = s->eng.ensureReady();
        if (st != MPM_OK) return st;
        st = s->eng.synchronize();
        if (st != MPM_OK) return st;
        *out = s.release();
        return MPM_OK;
    } catch (const std::bad_alloc&) {
        return mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
}

mpm_status mpm_solver_step(mpm_solver* s, int32_t nsteps) {
    MPM_TRY(check(s));
    GUARD(s->eng.step(nsteps));
}
mpm_status mpm_solver_synchronize(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.synchronize();
}
mpm_status mpm_solver_initialize(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.initialize(true);
}
mpm_status mpm_solver_reset_grid(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.resetGrid();
}
mpm_status mpm_solver_particles_to_grid(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.particlesToGrid();
}
mpm_status mpm_solver_compute_external_forces(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.gravity();
}
mpm_status mpm_solver_compute_gravity_forces(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.gravity();
}
mpm_status mpm_solver_update_grid_velocities(mpm_solver* s, float dt) {
    MPM_TRY(check(s));
    return s->eng.updateGridVelocities(dt);
}
mpm_status mpm_solver_grid_collision(mpm_solver* s, float dt) {
    MPM_TRY(check(s));
    return s->eng.gridCollision(dt);
}
mpm_status mpm_solver_solve_linear_system(mpm_solver* s, float dt) {
    MPM_TRY(check(s));
    return s->eng.solveLinearSystem(dt);  // a no-op while the solver is explicit (beta = 0), as in the reference
}
mpm_status mpm_solver_set_implicit(mpm_solver* s, float beta, int32_t max_iter, float tol) {
    MPM_TRY(check(s));
    return s->eng.setImplicit(s->scene, beta, max_iter, tol);
}
mpm_status mpm_solver_solve_info(mpm_solver* s, int32_t* iterations, float* residual) {
    MPM_TRY(check(s));
    return s->eng.solveInfo(s->scene, iterations, residual);
}
mpm_status mpm_solver_grid_to_particles(mpm_solver* s, float dt, float blend) {
    MPM_TRY(check(s));
    return s->eng.gridToParticles(dt, blend, true);
}
mpm_status mpm_solver_particles_collision(mpm_solver* s, float dt) {
    MPM_TRY(check(s));
    return s->eng.particlesCollision(dt);
}
mpm_status mpm_solver_advect_particles(mpm_solver* s, float dt) {
    MPM_TRY(check(s));
    return s->eng.advect(dt);
}
mpm_status mpm_solver_set_particles_collision(mpm_solver* s, int32_t enable) {
    MPM_TRY(check(s));
    return s->eng.setParticlesCollision(s->scene, enable);
}
mpm_status mpm_solver_set_level_set(mpm_solver* s, const float* phi, float friction, const float* velocity) {
    MPM_TRY(check(s));
    return s->eng.setLevelSet(s->scene, phi, friction, velocity);
}
mpm_status mpm_solver_set_cfl(mpm_solver* s, float cfl) {
    MPM_TRY(check(s));
    return s->eng.setCfl(s->scene, cfl);
}
mpm_status mpm_solver_time(mpm_solver* s, double* time, float* last_dt) {
    MPM_TRY(check(s));
    return s->eng.simTime(s->scene, time, last_dt);
}
mpm_status mpm_solver_get_particles_collision(const mpm_solver* s, int32_t* enable) {
    MPM_TRY(check(s));
    if (!enable) return mpm::fail(MPM_ERR_INVALID_ARG, "null output");
    *enable = const_cast<mpm_solver*>(s)->eng.scene(s->scene)->desc.particles_collision;
    return MPM_OK;
}
mpm_status mpm_solver_num_particles(const mpm_solver* s, size_t* n) {
    MPM_TRY(check(s));
    if (!n) return mpm::fail(MPM_ERR_INVALID_ARG, "null output");
    *n = const_cast<mpm_solver*>(s)->eng.scene(s->scene)->n;
    return MPM_OK;
}
mpm_status mpm_solver_get_desc(const mpm_solver* s, mpm_scene_desc* desc) {
    MPM_TRY(check(s));
    if (!desc) return mpm::fail(MPM_ERR_INVALID_ARG, "null output");
    *desc = const_cast<mpm_solver*>(s)->eng.scene(s->scene)->desc;
    return MPM_OK;
}
mpm_status mpm_solver_download(mpm_solver* s, int32_t field, float* host_out) {
    MPM_TRY(check(s));
    return s->eng.download(s->scene, field, host_out);
}
mpm_status mpm_solver_download_async(mpm_solver* s, int32_t field, float* host_out) {
    MPM_TRY(check(s));
    return s->eng.downloadAsync(s->scene, field, host_out);
}
mpm_status mpm_solver_download_wait(mpm_solver* s) {
    MPM_TRY(check(s));
    return s->eng.downloadWait();
}
mpm_status mpm_solver_download_density(mpm_solver* s, float* host_out) {
    MPM_TRY(check(s));
    return s->eng.downloadDensity(s->scene, host_out);
}
mpm_status mpm_solver_write_vdb(mpm_solver* s, const char* path) {
    MPM_TRY(check(s));
    if (!path) return mpm::fail(MPM_ERR_INVALID_ARG, "null path");
    try {
        const mpm_scene_desc& d = s->eng.scene(s->scene)->desc;
        std::vector<float> rho((size_t)d.resolution[0] * d.resolution[1] * d.resolution[2]);
        MPM_TRY(s->eng.downloadDensity(s->scene, rho.data()));
        return mpm::writeDensityVdb(rho.data(), d.resolution, path);
    } catch (const std::bad_alloc&) {
        return mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
}
mpm_status mpm_solver_download_grid(mpm_solver* s, int32_t field, float* host_out) {
    MPM_TRY(check(s));
    if (!host_out) return mpm::fail(MPM_ERR_INVALID_ARG, "null output");
    return s->eng.downloadGrid(s->scene, field, host_out);
}
mpm_status mpm_solver_upload(mpm_solver* s, int32_t field, const float* host_in) {
    MPM_TRY(check(s));
    return s->eng.upload(s->scene, field, host_in);
}
mpm_status mpm_solver_timed_step(mpm_solver* s, int32_t nsteps, float* ms) {
    MPM_TRY(check(s));
    GUARD(s->eng.timedStep(nsteps, ms));
}
mpm_status mpm_set_device(int32_t device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return mpm::fail(MPM_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    }
    return MPM_OK;
}
mpm_status mpm_release_cached_memory(int32_t device) {
    mpm_status st;
    cudaMemPool_t pool = mpm::scenePool(device, &st);
    if (!pool) return st;
    cudaError_t e = cudaMemPoolTrimTo(pool, 0);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return mpm::fail(MPM_ERR_CUDA, std::string("cudaMemPoolTrimTo: ") + cudaGetErrorString(e));
    }
    return MPM_OK;
}
mpm_status mpm_solver_stats(mpm_solver* s, mpm_step_stats* out) {
    MPM_TRY(check(s));
    return s->eng.stats(out);
}
mpm_status mpm_batch_stats(mpm_batch* b, mpm_step_stats* out) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.stats(out);
}
mpm_status mpm_solver_get_tuning(mpm_solver* s, mpm_tuning* out) {
    MPM_TRY(check(s));
    const mpm_scene_desc& d = s->eng.scene(s->scene)->desc;
    return s->eng.getTuning(d.interpolation, d.transfer, out);
}
mpm_status mpm_solver_set_tuning(mpm_solver* s, const mpm_tuning* t) {
    MPM_TRY(check(s));
    if (!t) return mpm::fail(MPM_ERR_INVALID_ARG, "null tuning");
    const mpm_scene_desc& d = s->eng.scene(s->scene)->desc;
    return s->eng.setTuning(d.interpolation, d.transfer, *t);
}
mpm_status mpm_solver_autotune(mpm_solver* s, int32_t steps_per_candidate, int32_t flags, int32_t* steps_run) {
    MPM_TRY(check(s));
    int run = 0;
    mpm_status st;
    try {
        st = s->eng.autotune(steps_per_candidate, flags, &run);
    } catch (const std::bad_alloc&) {
        st = mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
    if (steps_run) *steps_run = run;
    return st;
}
mpm_status mpm_batch_get_tuning(mpm_batch* b, int32_t interpolation, int32_t transfer, mpm_tuning* out) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.getTuning(interpolation, transfer, out);
}
mpm_status mpm_batch_set_tuning(mpm_batch* b, int32_t interpolation, int32_t transfer, const mpm_tuning* t) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    if (!t) return mpm::fail(MPM_ERR_INVALID_ARG, "null tuning");
    return b->eng.setTuning(interpolation, transfer, *t);
}
mpm_status mpm_batch_autotune(mpm_batch* b, int32_t steps_per_candidate, int32_t flags, int32_t* steps_run) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    int run = 0;
    mpm_status st;
    try {
        st = b->eng.autotune(steps_per_candidate, flags, &run);
    } catch (const std::bad_alloc&) {
        st = mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
    if (steps_run) *steps_run = run;
    return st;
}
mpm_status mpm_kernel_launches(uint64_t* count) {
    if (!count) return mpm::fail(MPM_ERR_INVALID_ARG, "null output");
    *count = mpm::kernelLaunches();
    return MPM_OK;
}
mpm_status mpm_solver_profile(mpm_solver* s, int32_t enable) {
    MPM_TRY(check(s));
    return s->eng.profile(enable);
}
mpm_status mpm_solver_profile_read(mpm_solver* s, float* ms, int32_t* counts, int32_t nfamilies) {
    MPM_TRY(check(s));
    return s->eng.profileRead(ms, counts, nfamilies);
}

mpm_status mpm_sort_keys(const uint32_t* keys, size_t n, int32_t bits, uint32_t* sorted_keys, uint32_t* perm) {
    if ((!keys || !sorted_keys || !perm) && n > 0) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    if (bits < 1 || bits > 32) return mpm::fail(MPM_ERR_INVALID_ARG, "bits must be in [1, 32]");
    if (n == 0) return MPM_OK;
    if (n > 0x7fffffffull) return mpm::fail(MPM_ERR_INVALID_ARG, "too many keys");
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return mpm::fail(MPM_ERR_CUDA, "mpm_sort_keys: no CUDA device");
    }
    mpm::DevMem k[2], v[2], scratch, err;
    mpm_status s = MPM_OK;
    for (int i = 0; i < 2 && s == MPM_OK; ++i) {
        s = k[i].alloc(sizeof(uint32_t) * n, "keys");
        if (s == MPM_OK) s = v[i].alloc(sizeof(uint32_t) * n, "values");
    }
    if (s == MPM_OK) s = scratch.alloc(sizeof(uint32_t) * mpm::onesweepScratchWords(n, bits), "sort scratch");
    if (s == MPM_OK) s = err.alloc(sizeof(uint32_t), "error flag");
    bool inB = false;
    uint32_t flag = 0;
    cudaError_t e = cudaSuccess;
    if (s == MPM_OK) {
        e = cudaMemsetAsync(err.p, 0, sizeof(uint32_t), st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(k[0].p, keys, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = mpm::radixSortOnesweep(k[0].as<uint32_t>(), v[0].as<uint32_t>(), k[1].as<uint32_t>(),
                                       v[1].as<uint32_t>(), n, bits, scratch.as<uint32_t>(), err.as<uint32_t>(), &inB,
                                       st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, err.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        const int r = inB ? 1 : 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sorted_keys, k[r].p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(perm, v[r].p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (s != MPM_OK) return s;
    if (e != cudaSuccess) return mpm::fail(MPM_ERR_CUDA, std::string("mpm_sort_keys: ") + cudaGetErrorString(e));
    if (flag) return mpm::fail(MPM_ERR_TIMEOUT, "mpm_sort_keys: a look-back wait gave up");
    return MPM_OK;
}

// ---- batch API (include/mpm_b200_batch.h) ----------------------------------
mpm_status mpm_batch_create(mpm_batch** out) {
    if (!out) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    std::unique_ptr<mpm_batch> b(new mpm_batch);
    mpm_status st = b->eng.init();
    if (st != MPM_OK) return st;
    *out = b.release();
    return MPM_OK;
}
mpm_status mpm_batch_destroy(mpm_batch* b) {
    if (!b) return MPM_OK;
    cudaStreamSynchronize(b->eng.stream());
    delete b;
    return MPM_OK;
}
mpm_status mpm_batch_add_scene(mpm_batch* b, const mpm_scene_desc* desc, const mpm_particles_in* particles,
                               int32_t* scene_id) {
    if (!b || !desc || !particles || !scene_id) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    int id = -1;
    mpm_status st = b->eng.addScene(*desc, *particles, &id);
    *scene_id = id;
    return st;
}
mpm_status mpm_batch_remove_scene(mpm_batch* b, int32_t scene_id) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.removeScene(scene_id);
}
mpm_status mpm_batch_save_scene(mpm_batch* b, int32_t scene_id, const char* path) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.saveScene(scene_id, path);
}
mpm_status mpm_batch_load_scene(mpm_batch* b, const char* path, int32_t* scene_id) {
    if (!b || !scene_id) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    try {
        Engine::Checkpoint ck;
        MPM_TRY(Engine::readCheckpoint(path, &ck));
        int id = -1;
        MPM_TRY(b->eng.loadScene(ck, &id));
        *scene_id = id;
        return MPM_OK;
    } catch (const std::bad_alloc&) {
        return mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
}
mpm_status mpm_batch_step(mpm_batch* b, int32_t nsteps) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    GUARD(b->eng.step(nsteps));
}
mpm_status mpm_solver_kernel_spans(mpm_solver* s, float* ms, int32_t* counts, int32_t nfamilies) {
    MPM_TRY(check(s));
    return s->eng.readSpans(ms, counts, nfamilies);
}
mpm_status mpm_batch_kernel_spans(mpm_batch* b, float* ms, int32_t* counts, int32_t nfamilies) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.readSpans(ms, counts, nfamilies);
}
mpm_status mpm_batch_time_steps(mpm_batch* b, int32_t enable) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.setStepTiming(enable != 0);
}
mpm_status mpm_batch_step_times(mpm_batch* b, float* ms, int32_t capacity, int32_t* count) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    int n = 0;
    mpm_status st = b->eng.stepTimes(ms, capacity, &n);
    if (count) *count = n;
    return st;
}
mpm_status mpm_batch_wait_steps(mpm_batch* b, int32_t in_flight) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.waitSteps(in_flight);
}
mpm_status mpm_batch_synchronize(mpm_batch* b) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.synchronize();
}
mpm_status mpm_batch_download(mpm_batch* b, int32_t scene_id, int32_t field, float* host_out) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.download(scene_id, field, host_out);
}
mpm_status mpm_batch_download_async(mpm_batch* b, int32_t scene_id, int32_t field, float* host_out) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.downloadAsync(scene_id, field, host_out);
}
mpm_status mpm_batch_download_wait(mpm_batch* b) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.downloadWait();
}
mpm_status mpm_batch_download_density(mpm_batch* b, int32_t scene_id, float* host_out) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.downloadDensity(scene_id, host_out);
}
mpm_status mpm_batch_write_vdb(mpm_batch* b, int32_t scene_id, const char* path) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    if (!path) return mpm::fail(MPM_ERR_INVALID_ARG, "null path");
    try {
        const mpm::SceneHost* sc = b->eng.scene(scene_id);
        if (!sc) return mpm::fail(MPM_ERR_INVALID_ARG, "unknown scene id");
        const mpm_scene_desc d = sc->desc;
        std::vector<float> rho((size_t)d.resolution[0] * d.resolution[1] * d.resolution[2]);
        MPM_TRY(b->eng.downloadDensity(scene_id, rho.data()));
        return mpm::writeDensityVdb(rho.data(), d.resolution, path);
    } catch (const std::bad_alloc&) {
        return mpm::fail(MPM_ERR_OOM, "host allocation failed");
    }
}
mpm_status mpm_batch_set_level_set(mpm_batch* b, int32_t scene_id, const float* phi, float friction,
                                   const float* velocity) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.setLevelSet(scene_id, phi, friction, velocity);
}
mpm_status mpm_batch_set_implicit(mpm_batch* b, int32_t scene_id, float beta, int32_t max_iter, float tol) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.setImplicit(scene_id, beta, max_iter, tol);
}
mpm_status mpm_batch_solve_info(mpm_batch* b, int32_t scene_id, int32_t* iterations, float* residual) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.solveInfo(scene_id, iterations, residual);
}
mpm_status mpm_batch_set_cfl(mpm_batch* b, int32_t scene_id, float cfl) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.setCfl(scene_id, cfl);
}
mpm_status mpm_batch_time(mpm_batch* b, int32_t scene_id, double* time, float* last_dt) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.simTime(scene_id, time, last_dt);
}
mpm_status mpm_batch_num_scenes(const mpm_batch* b, int32_t* n) {
    if (!b || !n) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    *n = (int32_t)b->eng.numScenes();
    return MPM_OK;
}
mpm_status mpm_batch_scene_particles(const mpm_batch* b, int32_t scene_id, size_t* n) {
    if (!b || !n) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    const mpm::SceneHost* s = const_cast<mpm_batch*>(b)->eng.scene(scene_id);
    if (!s) return mpm::fail(MPM_ERR_INVALID_ARG, "unknown scene id");
    *n = s->n;
    return MPM_OK;
}
mpm_status mpm_batch_scene_desc(const mpm_batch* b, int32_t scene_id, mpm_scene_desc* desc) {
    if (!b || !desc) return mpm::fail(MPM_ERR_INVALID_ARG, "null argument");
    const mpm::SceneHost* s = const_cast<mpm_batch*>(b)->eng.scene(scene_id);
    if (!s) return mpm::fail(MPM_ERR_INVALID_ARG, "unknown scene id");
    *desc = s->desc;
    return MPM_OK;
}
mpm_status mpm_batch_timed_step(mpm_batch* b, int32_t nsteps, float* ms) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    GUARD(b->eng.timedStep(nsteps, ms));
}
mpm_status mpm_batch_profile(mpm_batch* b, int32_t enable) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.profile(enable);
}
mpm_status mpm_batch_profile_read(mpm_batch* b, float* ms, int32_t* counts, int32_t nfamilies) {
    if (!b) return mpm::fail(MPM_ERR_INVALID_ARG, "null batch");
    return b->eng.profileRead(ms, counts, nfamilies);
}

}  // extern "C"
