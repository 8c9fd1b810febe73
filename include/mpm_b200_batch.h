/*
 * mpm_b200_batch.h -- batched scenes on one GPU.
 *
 * The reference advances exactly one scene per solver object
 * (chains::MPMSolver3D, include/mpm_solver3d.h:21-96) and has no batching;
 * these entry points have no counterpart in the reference.  A batch advances
 * many independent scenes of different particle counts, grids, transfers and
 * materials with one launch sequence per step (sort, P2G, grid, G2P over the
 * active grid blocks of every scene).  Scenes may be added and removed
 * between steps, which the serving loop uses for continuous batching.
 */
#ifndef MPM_B200_BATCH_H_
#define MPM_B200_BATCH_H_

#include "mpm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mpm_batch mpm_batch;

MPM_API mpm_status mpm_batch_create(mpm_batch** out);
MPM_API mpm_status mpm_batch_destroy(mpm_batch* b);
/* Upload a scene (initialized on the next step); returns its id. */
MPM_API mpm_status mpm_batch_add_scene(mpm_batch* b, const mpm_scene_desc* desc,
                               const mpm_particles_in* particles, int32_t* scene_id);
/* Release a scene's device state (returned to the memory pool after the
 * batch's queued steps; does not wait for them). */
MPM_API mpm_status mpm_batch_remove_scene(mpm_batch* b, int32_t scene_id);
/* Checkpoint one scene of a batch / add a scene from a checkpoint (the
 * format of mpm_solver_save; a scene saved from a solver or a batch loads into
 * either).  For preempting and resuming served requests. */
MPM_API mpm_status mpm_batch_save_scene(mpm_batch* b, int32_t scene_id, const char* path);
MPM_API mpm_status mpm_batch_load_scene(mpm_batch* b, const char* path, int32_t* scene_id);
/* Advance every scene nsteps steps (asynchronous). */
MPM_API mpm_status mpm_batch_step(mpm_batch* b, int32_t nsteps);
MPM_API mpm_status mpm_batch_synchronize(mpm_batch* b);
/* Per-step device times for a serving loop that does not synchronize every
 * step.  With timing on (enable = 1), every step is bracketed by two events;
 * mpm_batch_step_times returns, without waiting, the device times (ms) of up
 * to `capacity` steps that have completed, oldest first, in *count;
 * mpm_batch_wait_steps blocks until at most `in_flight` timed steps are still
 * queued or running (1 keeps the next step queued behind the running one). */
MPM_API mpm_status mpm_batch_time_steps(mpm_batch* b, int32_t enable);
MPM_API mpm_status mpm_batch_step_times(mpm_batch* b, float* ms, int32_t capacity, int32_t* count);
MPM_API mpm_status mpm_batch_wait_steps(mpm_batch* b, int32_t in_flight);
/* Download a particle field of one scene in its original particle order. */
MPM_API mpm_status mpm_batch_download(mpm_batch* b, int32_t scene_id, int32_t field, float* host_out);
/* Asynchronous form (see mpm_solver_download_async) and its wait. */
MPM_API mpm_status mpm_batch_download_async(mpm_batch* b, int32_t scene_id, int32_t field, float* host_out);
MPM_API mpm_status mpm_batch_download_wait(mpm_batch* b);
/* Density grid of one scene (see mpm_solver_download_density). */
MPM_API mpm_status mpm_batch_download_density(mpm_batch* b, int32_t scene_id, float* host_out);
/* OpenVDB file of one scene's density grid (see mpm_solver_write_vdb). */
MPM_API mpm_status mpm_batch_write_vdb(mpm_batch* b, int32_t scene_id, const char* path);
/* Semi-implicit update of one scene (see mpm_solver_set_implicit). */
MPM_API mpm_status mpm_batch_set_implicit(mpm_batch* b, int32_t scene_id, float beta, int32_t max_iter, float tol);
MPM_API mpm_status mpm_batch_solve_info(mpm_batch* b, int32_t scene_id, int32_t* iterations, float* residual);
/* CFL time step and simulated time of one scene (see mpm_solver_set_cfl,
 * mpm_solver_time). */
MPM_API mpm_status mpm_batch_set_cfl(mpm_batch* b, int32_t scene_id, float cfl);
MPM_API mpm_status mpm_batch_time(mpm_batch* b, int32_t scene_id, double* time, float* last_dt);
/* Level-set collision object of one scene (see mpm_solver_set_level_set). */
MPM_API mpm_status mpm_batch_set_level_set(mpm_batch* b, int32_t scene_id, const float* phi, float friction,
                                           const float* velocity);
MPM_API mpm_status mpm_batch_num_scenes(const mpm_batch* b, int32_t* n);
MPM_API mpm_status mpm_batch_scene_particles(const mpm_batch* b, int32_t scene_id, size_t* n);
MPM_API mpm_status mpm_batch_scene_desc(const mpm_batch* b, int32_t scene_id, mpm_scene_desc* desc);
MPM_API mpm_status mpm_batch_stats(mpm_batch* b, mpm_step_stats* out);
/* Launch settings (see mpm_tuning) of the batch's scenes of one
 * (interpolation, transfer) combination; -1 in either selects every value
 * (set) -- get needs both.  Combinations not set use the defaults. */
MPM_API mpm_status mpm_batch_get_tuning(mpm_batch* b, int32_t interpolation, int32_t transfer, mpm_tuning* out);
MPM_API mpm_status mpm_batch_set_tuning(mpm_batch* b, int32_t interpolation, int32_t transfer, const mpm_tuning* t);
/* Autotuner (see mpm_solver_autotune), per (interpolation, transfer,
 * particles-per-cell bucket) key of each combination in the batch: the batch's
 * steps time every combination at once. */
MPM_API mpm_status mpm_batch_autotune(mpm_batch* b, int32_t steps_per_candidate, int32_t flags, int32_t* steps_run);
/* nsteps steps bracketed by events on the batch's stream; device ms in *ms. */
MPM_API mpm_status mpm_batch_timed_step(mpm_batch* b, int32_t nsteps, float* ms);
/* Kernel spans of the batch's steps (see mpm_solver_kernel_spans). */
MPM_API mpm_status mpm_batch_kernel_spans(mpm_batch* b, float* ms, int32_t* counts, int32_t nfamilies);
MPM_API mpm_status mpm_batch_profile(mpm_batch* b, int32_t enable);
MPM_API mpm_status mpm_batch_profile_read(mpm_batch* b, float* ms, int32_t* counts, int32_t nfamilies);

#ifdef __cplusplus
}
#endif

#endif /* MPM_B200_BATCH_H_ */
