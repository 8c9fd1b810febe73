/*
 * mpm_b200.h -- C ABI of the B200-native MPM snow step.
 *
 * This is the drop-in boundary for the particle step of H-YWu/mpm
 * (chains::MPMSolver3D / chains::APICMPMSolver3D).  Every entry point takes
 * plain pointers and sizes; no CUDA, Eigen or torch type crosses it.  Each
 * declaration names the reference interface it replaces (file:line inside the
 * reference project).
 *
 * Conventions
 *  - Every call returns an mpm_status.  Nothing in the library calls exit();
 *    mpm_last_error_string() returns a message for the calling thread.
 *  - Host arrays of 3-vectors are interleaved (x0,y0,z0,x1,...), matching the
 *    Eigen::Vector3f layout of the reference's particles.
 *  - Particle downloads are returned in the caller's original particle order,
 *    although the device keeps particles sorted by grid cell.
 *  - A solver handle is single-threaded; each handle owns one CUDA stream.
 */
#ifndef MPM_B200_H_
#define MPM_B200_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MPM_API __attribute__((visibility("default")))
#else
#define MPM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MPM_B200_ABI_VERSION 1

/* Status codes.  The reference prints and calls exit() on CUDA errors
 * (include/cuda_utils.h:6-20) and throws std::runtime_error on bad enums
 * (src/mpm3d_parser.cpp:10,17); here both become return codes. */
typedef enum mpm_status {
    MPM_OK = 0,
    MPM_ERR_INVALID_ARG = 1,
    MPM_ERR_IO = 2,
    MPM_ERR_PARSE = 3,
    MPM_ERR_OOM = 4,
    MPM_ERR_CUDA = 5,
    MPM_ERR_NUMERIC = 6,   /* NaN/Inf particle state detected on the device */
    MPM_ERR_BUDGET = 7,    /* device-memory budget of a batch exceeded       */
    MPM_ERR_TIMEOUT = 8,
    MPM_ERR_UNSUPPORTED = 9
} mpm_status;

/* chains::InterpolationType (include/enums.h:6-10) */
enum {
    MPM_INTERP_LINEAR = 0,
    MPM_INTERP_QUADRATIC_BSPLINE = 1,
    MPM_INTERP_CUBIC_BSPLINE = 2
};

/* chains::ConstitutiveModel (include/enums.h:12-15) */
enum {
    MPM_MODEL_FIXED_COROTATED = 0,
    MPM_MODEL_NEO_HOOKEAN = 1
};

/* Transfer scheme: MPMSolver3D (PIC-FLIP, include/mpm_solver3d.h:21) or
 * APICMPMSolver3D (include/apic_mpm_solver3d.h:20). */
enum {
    MPM_TRANSFER_PIC_FLIP = 0,
    MPM_TRANSFER_APIC = 1
};

/* Grid boundary condition.
 *  REFERENCE: applyBoundaryCollision on the grid box at the node's
 *             "distorted" position x_i + dt v*_i (src/mpm_solver3d.cu:405-426,
 *             src/collision_object3d.cu:7-54).
 *  STICKY:    v* = 0 on nodes within `sticky_cells` of any grid face. */
enum {
    MPM_BOUNDARY_REFERENCE = 0,
    MPM_BOUNDARY_STICKY = 1
};

/* Initial particle volume.
 *  GRID_ESTIMATE: V0 = m / (sum_i m_i w_ip / h^3), as the reference's
 *                 initialize() does (src/mpm_solver3d.cu:131-223).
 *  PRESCRIBED:    V0 taken from mpm_particles_in.volume. */
enum {
    MPM_VOLUME_GRID_ESTIMATE = 0,
    MPM_VOLUME_PRESCRIBED = 1
};

/* Per-group material.  Lame parameters are derived exactly as the
 * reference's particle constructor does (src/material_point3d.cu:25-26). */
typedef struct mpm_material {
    float youngs_modulus;
    float poisson_ratio;
    float hardening;             /* xi      */
    float critical_compression;  /* theta_c */
    float critical_stretch;      /* theta_s */
    int32_t model;               /* MPM_MODEL_* */
} mpm_material;

/* Scene description: the arguments of the reference's solver constructors
 * (include/mpm_solver3d.h:25-34, include/apic_mpm_solver3d.h:24-32) plus the
 * options the benchmark scenes need. */
typedef struct mpm_scene_desc {
    float origin[3];
    int32_t resolution[3];
    float stride;                /* grid spacing h                              */
    float friction;              /* boundary friction coefficient               */
    float blend;                 /* FLIP weight alpha (PIC-FLIP only)           */
    float dt;                    /* fixed time step                             */
    float gravity;               /* |g| along -y; the reference hard-codes 9.80665 */
    int32_t transfer;            /* MPM_TRANSFER_*                              */
    int32_t interpolation;       /* MPM_INTERP_*                                */
    int32_t boundary;            /* MPM_BOUNDARY_*                              */
    int32_t sticky_cells;        /* wall thickness in cells for STICKY          */
    int32_t volume_mode;         /* MPM_VOLUME_*                                */
    int32_t particles_collision; /* initial _enable_particles_collision (0/1)   */
} mpm_scene_desc;

/* Host-side particle input.  Replaces thrust::host_vector<MaterialPoint3D>
 * (include/material_point3d.h:14-22); the per-particle material constants
 * of the reference become an index into `materials`. */
typedef struct mpm_particles_in {
    size_t n;
    const float* position;       /* 3n, interleaved                  */
    const float* velocity;       /* 3n, interleaved                  */
    const float* mass;           /* n                                */
    const uint16_t* material;    /* n, may be NULL if nmaterials == 1 */
    const float* volume;         /* n, only read for VOLUME_PRESCRIBED */
    const mpm_material* materials;
    int32_t nmaterials;
} mpm_particles_in;

/* Particle fields for mpm_solver_download (floats per particle). */
enum {
    MPM_FIELD_POSITION = 0,          /* 3 */
    MPM_FIELD_VELOCITY = 1,          /* 3 */
    MPM_FIELD_FE = 2,                /* 9, row-major */
    MPM_FIELD_FP = 3,                /* 9, row-major */
    MPM_FIELD_B = 4,                 /* 9, row-major, APIC only */
    MPM_FIELD_VOLUME0 = 5,           /* 1 */
    MPM_FIELD_MASS = 6,              /* 1 */
    MPM_FIELD_POSITION4 = 7,         /* 4: (x, y, z, 1), the headless VBO export */
    MPM_FIELD_DET_FE = 8,            /* 1 */
    MPM_FIELD_DET_FP = 9             /* 1 */
};

/* Dense grid fields for mpm_solver_download_grid (floats per node, node
 * index x + X*(y + Y*z) as in src/mpm_solver3d.cu:257). */
enum {
    MPM_GRID_MASS = 0,               /* 1 */
    MPM_GRID_VELOCITY = 1,           /* 3: momentum after P2G, v after update */
    MPM_GRID_FORCE = 2,              /* 3 */
    MPM_GRID_VELOCITY_STAR = 3       /* 3 */
};

typedef struct mpm_solver mpm_solver;

/* Library version / capability query. */
MPM_API int32_t mpm_abi_version(void);
/* Message for the last failing call on this thread ("" if none). */
MPM_API const char* mpm_last_error_string(void);
/* Number of CUDA devices visible (0 on a host without a GPU). */
MPM_API mpm_status mpm_device_count(int32_t* count);
/* Select the CUDA device that later solver/batch creations on this thread
 * use (the library's CUDA runtime keeps its own current device). */
MPM_API mpm_status mpm_set_device(int32_t device);
/* Scene state (particle buffers, grids, download staging) comes from a
 * per-device stream-ordered memory pool that keeps freed memory for the next
 * scene, so adding and removing scenes needs no cudaMalloc/cudaFree.  This
 * returns the pool's unused memory on `device` to the driver.  No
 * counterpart in the reference (thrust::device_vector allocates per
 * solver). */
MPM_API mpm_status mpm_release_cached_memory(int32_t device);

/* Counters of the last step (read back from the device; synchronizes). */
typedef struct mpm_step_stats {
    uint32_t active_blocks;    /* 4^3-cell blocks holding particles          */
    uint32_t outside_blocks;   /* scenes with particles whose stencil misses the grid */
    uint32_t active_nodes;     /* grid nodes with non-zero mass              */
    uint32_t reserved;
} mpm_step_stats;

/* Construct a solver on the current CUDA device, upload the particles and
 * run initialize().  Replaces MPMSolver3D::MPMSolver3D
 * (src/mpm_solver3d.cu:36-91) and APICMPMSolver3D::APICMPMSolver3D
 * (src/apic_mpm_solver3d.cu:36-90). */
MPM_API mpm_status mpm_solver_create(const mpm_scene_desc* desc,
                             const mpm_particles_in* particles,
                             mpm_solver** out);
/* Replaces ~MPMSolver3D (src/mpm_solver3d.cu:93-98). */
MPM_API mpm_status mpm_solver_destroy(mpm_solver* s);

/* Checkpoint and resume (no counterpart in the reference, which has no
 * checkpoint).  mpm_solver_save writes the scene description, the material
 * table and the full particle state -- every field, in the solver's internal
 * particle order, with the cached stress -- to `path`; mpm_solver_load creates
 * a solver from such a file (checked on the host before any device work:
 * MPM_ERR_IO if unreadable, MPM_ERR_PARSE if not a valid checkpoint).  The
 * loaded solver's steps are bitwise those the saved solver would have taken. */
MPM_API mpm_status mpm_solver_save(mpm_solver* s, const char* path);
MPM_API mpm_status mpm_solver_load(const char* path, mpm_solver** out);

/* simulateOneStep() repeated nsteps times (src/mpm_solver3d.cu:100-125,
 * src/apic_mpm_solver3d.cu:99-124).  Asynchronous on the solver's stream;
 * returns errors of earlier steps. */
MPM_API mpm_status mpm_solver_step(mpm_solver* s, int32_t nsteps);
/* Wait for the solver's stream; reports MPM_ERR_NUMERIC if a non-finite
 * particle state was seen since the last call. */
MPM_API mpm_status mpm_solver_synchronize(mpm_solver* s);

/* Sub-steps of simulateOneStep, run in split (unfused) form for testing and
 * for callers that drive the step themselves
 * (include/mpm_solver3d.h:40-63, include/apic_mpm_solver3d.h:38-61). */
MPM_API mpm_status mpm_solver_initialize(mpm_solver* s);                  /* :131-223 */
MPM_API mpm_status mpm_solver_reset_grid(mpm_solver* s);                  /* :225-235 */
MPM_API mpm_status mpm_solver_particles_to_grid(mpm_solver* s);           /* :237-294 */
MPM_API mpm_status mpm_solver_compute_external_forces(mpm_solver* s);     /* :296-298 */
MPM_API mpm_status mpm_solver_compute_gravity_forces(mpm_solver* s);      /* :394-403 */
MPM_API mpm_status mpm_solver_update_grid_velocities(mpm_solver* s, float dt);   /* :300-310 */
MPM_API mpm_status mpm_solver_grid_collision(mpm_solver* s, float dt);    /* :405-426 */
MPM_API mpm_status mpm_solver_solve_linear_system(mpm_solver* s, float dt);      /* :312-314, see below */
MPM_API mpm_status mpm_solver_grid_to_particles(mpm_solver* s, float dt, float blend); /* :316-379 */
MPM_API mpm_status mpm_solver_particles_collision(mpm_solver* s, float dt);      /* :428-445 */
MPM_API mpm_status mpm_solver_advect_particles(mpm_solver* s, float dt);  /* :381-391 */

/* _enable_particles_collision and switchIfEnableParticlesCollision()
 * (include/mpm_solver3d.h:23,40, src/mpm_solver3d.cu:127-129). */
MPM_API mpm_status mpm_solver_set_particles_collision(mpm_solver* s, int32_t enable);
MPM_API mpm_status mpm_solver_get_particles_collision(const mpm_solver* s, int32_t* enable);

/* Level-set collision object (LevelSetCollisionObject3D, a level set per grid
 * node, include/collision_object3d.h:9-12; declared but never applied by the
 * reference).  phi: res_x*res_y*res_z signed distances in world units at the
 * grid nodes, index x + X*(y + Y*z), negative inside the object; NULL removes
 * the object.  Each grid collision (and each particle collision when enabled)
 * applies it after the grid boundary: the distance is interpolated
 * trilinearly at the moved position (node + dt v*, particle + dt v); where it
 * is <= 0 the velocity relative to the object's surface velocity gets the
 * friction law of applyBoundaryCollision (src/collision_object3d.cu:38-51)
 * with the normalised trilinear gradient as normal.  velocity (3 floats, NULL
 * = at rest) is the surface velocity; friction >= 0.  The values are copied. */
MPM_API mpm_status mpm_solver_set_level_set(mpm_solver* s, const float* phi, float friction, const float* velocity);

/* Semi-implicit update (IntegrationType SEMI_IMPLICIT / FULL_IMPLICIT,
 * include/enums.h:17-21, and solveLinearSystem, src/mpm_solver3d.cu:312-314:
 * declared, left empty by the reference).  beta > 0 makes every step solve
 * (M + beta dt^2 H) v = M v* after the grid collision, H the Hessian of the
 * elastic energy in the node positions (Stomakhin et al. 2013, section 9),
 * by conjugate residual preconditioned with the node masses, to
 * |r| <= tol |M v*| or max_iter iterations, then apply the grid collision to
 * the solved velocities; beta = 1/2 is the semi-implicit, 1 the backward
 * Euler update, 0 the explicit step.  mpm_solver_solve_linear_system then
 * runs the same solve on the split-mode grid (no collision after). */
MPM_API mpm_status mpm_solver_set_implicit(mpm_solver* s, float beta, int32_t max_iter, float tol);
/* Iterations and final |r| / |M v*| of the last solve (waits for the queued work). */
MPM_API mpm_status mpm_solver_solve_info(mpm_solver* s, int32_t* iterations, float* residual);

/* CFL time step (listed as unimplemented in the reference, README.md:60-67).
 * cfl > 0: every mpm_solver_step step takes dt = min(desc.dt, cfl * stride /
 * max_p |v_p|), from the particle velocities the step starts with, computed
 * on the device (no host round trip); cfl = 0 returns to the fixed desc.dt.
 * The sub-step functions keep the dt they are given. */
MPM_API mpm_status mpm_solver_set_cfl(mpm_solver* s, float cfl);
/* Simulated time advanced by mpm_solver_step since creation (carried by
 * checkpoints) and the dt of the last step; either pointer may be NULL.
 * Waits for the queued steps. */
MPM_API mpm_status mpm_solver_time(mpm_solver* s, double* time, float* last_dt);

MPM_API mpm_status mpm_solver_num_particles(const mpm_solver* s, size_t* n);
MPM_API mpm_status mpm_solver_get_desc(const mpm_solver* s, mpm_scene_desc* desc);

/* Download a particle field in the original particle order.  `host_out`
 * holds n * floats-per-particle floats.  MPM_FIELD_POSITION4 replaces the
 * GL buffer export (src/mpm_solver3d.cu:447-508). */
MPM_API mpm_status mpm_solver_download(mpm_solver* s, int32_t field, float* host_out);
/* Asynchronous download of the current state (same layout as
 * mpm_solver_download): the device gather runs in the solver's stream order,
 * the copy into host_out runs on a copy stream and overlaps later steps.
 * Returns at once; host_out (pinned memory for the copy to overlap) must stay
 * valid and unread until mpm_solver_download_wait or mpm_solver_synchronize
 * returns.  Two staging buffers alternate, so any number of downloads may be
 * queued; the third waits on the device for the first one's copy.  No
 * counterpart in the reference, whose per-frame export
 * (updateGLBufferWithCUDA, src/mpm_solver3d.cu:447-508) copies synchronously. */
MPM_API mpm_status mpm_solver_download_async(mpm_solver* s, int32_t field, float* host_out);
/* Wait for every asynchronous download issued so far. */
MPM_API mpm_status mpm_solver_download_wait(mpm_solver* s);
/* Density of the current state on the dense grid: res[0]*res[1]*res[2]
 * floats, node index x + X (y + Y z), value sum_p m_p w_ip / h^3 -- the grid
 * that writeToOpenVDB (src/mpm_solver3d.cu:509-572) rasterises and writes as
 * an OpenVDB "density" grid; here it is returned headless (no OpenVDB file).
 * Does not change the particle state. */
MPM_API mpm_status mpm_solver_download_density(mpm_solver* s, float* host_out);

/* Write the density grid of the current state (mpm_solver_download_density)
 * as an OpenVDB file: one FloatGrid named "density", background 0, the
 * reference's default transform (voxel size 1: a voxel is a grid node
 * index), the nodes with non-zero density active, in the standard 5-4-3 tree
 * of 8^3 leaves (file format version 224, active-mask compression, no zip or
 * blosc).  Replaces MPMSolver3D::writeToOpenVDB (include/mpm_solver3d.h:74,
 * src/mpm_solver3d.cu:509-572), which needs the OpenVDB library; this writes
 * the format directly. */
MPM_API mpm_status mpm_solver_write_vdb(mpm_solver* s, const char* path);
/* The same file from a caller's dense density array (res[0] x res[1] x res[2]
 * floats, index x + X (y + Y z)); host only, no device work. */
MPM_API mpm_status mpm_write_vdb_density(const float* density, const int32_t* resolution, const char* path);
/* Download a dense grid field (res^3 * components floats).  Valid after
 * particles_to_grid() and the grid sub-steps of the split API, or after
 * mpm_solver_step when the solver keeps the dense debug grid. */
MPM_API mpm_status mpm_solver_download_grid(mpm_solver* s, int32_t field, float* host_out);

/* Overwrite the particle state (original order) with host data of the same
 * layout as mpm_solver_download; marks cached stress as stale. */
MPM_API mpm_status mpm_solver_upload(mpm_solver* s, int32_t field, const float* host_in);

/* Stable device radix sort of n 32-bit keys by their low `bits` bits, the
 * sort every step runs on particle cell keys (no counterpart in the
 * reference, which scatters unsorted with atomics).  Outputs the sorted keys
 * and, for each sorted position, the input index.  Host buffers; used to
 * check the sort bit-exactly against a CPU stable sort. */
MPM_API mpm_status mpm_sort_keys(const uint32_t* keys, size_t n, int32_t bits, uint32_t* sorted_keys,
                                 uint32_t* perm);

/* The same stable sort for callers that cannot allocate device memory: no
 * counterpart in the reference.  Some callers own all device memory
 * themselves -- a host application with its own pool or a budget fixed at
 * start-up, or a loop that must not risk the implicit device synchronization
 * of cudaMalloc/cudaFree -- and hand the library only buffers they allocated.
 * Here `keys` (n inputs, only read), `sorted_keys` and `perm` (n outputs)
 * are device pointers from the caller, `stream` is a cudaStream_t (NULL for
 * the default stream), and the call is asynchronous on that stream.  The
 * call allocates nothing: its working memory is one fixed device array
 * inside the library that every GPU loading the library keeps until the
 * process exits.  Limits: n <= MPM_SORT_NOALLOC_MAX_KEYS (larger n is
 * rejected with MPM_ERR_INVALID_ARG); all calls share the array, so calls
 * that overlap on the GPU race -- keep them on one stream.  The three buffers
 * must not overlap (an in-place sort is rejected with MPM_ERR_INVALID_ARG).
 * The call works on the current device (mpm_set_device): `stream` must
 * belong to it, else MPM_ERR_INVALID_ARG.  The first call on each device
 * resolves the array's device address (cudaGetSymbolAddress) and caches it
 * for the process, so make that first call during set-up, and do not call
 * across a cudaDeviceReset of that device. */
#define MPM_SORT_NOALLOC_MAX_KEYS (1u << 20)
MPM_API mpm_status mpm_sort_keys_device_noalloc(const uint32_t* keys, uint32_t n, int32_t bits,
                                                uint32_t* sorted_keys, uint32_t* perm, void* stream);

/* Run nsteps steps bracketed by CUDA events recorded on the solver's own
 * stream and return the device time in *ms (synchronizes).  Used by the
 * benchmark; same work as mpm_solver_step. */
MPM_API mpm_status mpm_solver_timed_step(mpm_solver* s, int32_t nsteps, float* ms);

MPM_API mpm_status mpm_solver_stats(mpm_solver* s, mpm_step_stats* out);

/* Launch settings of the step kernels (no counterpart in the reference, whose
 * thrust launches run one thread per particle or node).  They decide how the
 * work is spread over the GPU and never the order of any sum, so every result
 * is bitwise the same for any setting.
 *   g2p_chunk:    particles per G2P work item, MPM_G2P_CHUNK_MIN..MPM_G2P_CHUNK_MAX
 *                 (a grid block's particles are split into items of this size);
 *   p2g_stage:    particles staged per P2G warp pass, 16, 24 or 32 (0: chosen
 *                 from the particle density after the first step);
 *   p2g_warp_max: P2G work items of at most this many particles are taken by
 *                 single warps instead of whole CTAs, 0..MPM_P2G_WARP_MAX_MAX
 *                 (0: none; -1: the engine's choice -- items of at most 256
 *                 particles, taken by warps in a step where their
 *                 (stencil, transfer) combination has at least 1024 of them,
 *                 decided on the device each step). */
typedef struct mpm_tuning {
    int32_t g2p_chunk;
    int32_t p2g_stage;
    int32_t p2g_warp_max;
} mpm_tuning;
#define MPM_P2G_WARP_MAX_MAX 4096
#define MPM_G2P_CHUNK_MIN 256
#define MPM_G2P_CHUNK_MAX 4096

MPM_API mpm_status mpm_solver_get_tuning(mpm_solver* s, mpm_tuning* out);
MPM_API mpm_status mpm_solver_set_tuning(mpm_solver* s, const mpm_tuning* t);

/* Autotuner of the launch settings.  The key of a scene is its stencil
 * (interpolation), its transfer and its bucket of particles per occupied cell
 * (< 2, < 8, < 32, >= 32), measured by one step.  A key found in the tuning
 * cache (this process's, then the per-device cache file) takes the cached
 * settings; otherwise every G2P chunk of {256, 512, 1024, 2048, 4096} and
 * every P2G staging size of {16, 24, 32} is timed with CUDA events around the
 * P2G and G2P launches of each combination (one combination after another)
 * over `steps_per_candidate` steps (after one untimed step each) and the fastest
 * of each is kept and cached; the P2G warp threshold stays the engine's
 * choice (-1).  The tuning steps
 * are real steps of the simulation (they advance it; their results are those
 * of any other settings); *steps_run (may be NULL) returns how many were
 * taken.  The cache file is $MPM_TUNE_CACHE, else
 * $XDG_CACHE_HOME/mpm_b200/tuning.txt, else ~/.cache/mpm_b200/tuning.txt.
 * flags: MPM_TUNE_FORCE measures even cached keys; MPM_TUNE_NO_DISK neither
 * reads nor writes the file. */
#define MPM_TUNE_FORCE 1
#define MPM_TUNE_NO_DISK 2
MPM_API mpm_status mpm_solver_autotune(mpm_solver* s, int32_t steps_per_candidate, int32_t flags,
                                       int32_t* steps_run);

/* Total kernel launches issued by this library in this process. */
MPM_API mpm_status mpm_kernel_launches(uint64_t* count);

/* Timing of the solver's kernels: fills ms[k] with the average device time
 * of kernel family k over the last timed steps (see mpm_solver_profile). */
/* Device-measured kernel times inside the ordinary (graph-replayed) step:
 * for the families P2G, grid and G2P (k = 0, 1, 2) the time from the first
 * CTA's start to the last CTA's end of each launch (%globaltimer), averaged
 * per step since the last call (summed over the stencil/transfer
 * combinations of a batch), and the number of steps; the counters restart.
 * No counterpart in the reference. */
MPM_API mpm_status mpm_solver_kernel_spans(mpm_solver* s, float* ms, int32_t* counts, int32_t nfamilies);
MPM_API mpm_status mpm_solver_profile(mpm_solver* s, int32_t enable);
MPM_API mpm_status mpm_solver_profile_read(mpm_solver* s, float* ms, int32_t* counts, int32_t nfamilies);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_H_ */
