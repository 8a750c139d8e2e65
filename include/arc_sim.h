/*
 * arc_sim.h - C ABI of the B200 batched world step (libarcsim.so).
 *
 * Part 1 is the reference's batched API, symbol for symbol, so that the
 * reference's ctypes binding (arc/native.py:38-55) and its C callers load
 * this library unchanged. Every call there keeps the reference's contract:
 * host float64 / int32 buffers, synchronous (results are in the caller's
 * buffers when the call returns), void returns, NULL only from create.
 *
 * Part 2 is additive: status codes, precision and kernel selection, state
 * snapshots, per-world terrain, custom models for the analytic scenes, and
 * the device-resident path (device pointers, an explicit CUDA stream).
 *
 * All functions have C linkage and plain pointer/size arguments; none takes
 * a PyTorch or CUDA runtime type (streams are passed as void *).
 */
#ifndef ARC_SIM_H
#define ARC_SIM_H

#include "arc_world.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct arc_sim arc_sim;

/* Sizes of the per-world blocks of arc_sim_observe (csrc/arc_sim.h:17-21). */
#define ARC_SIM_ROOT_SIZE 13    /* pos(3) quat wxyz(4) linvel(3) angvel(3), world frame */
#define ARC_SIM_ROT_SIZE 9      /* torso rotation matrix (body to world), row-major */
#define ARC_SIM_JOINT_SIZE 36   /* angles, rates, torques */
#define ARC_SIM_CONTACT_SIZE 6  /* feet, torso, other leg parts */

/* ======================================================================
 * Part 1: the reference API (csrc/arc_sim.h:25-56)
 * ====================================================================== */

/* Replaces csrc/arc_sim.h:25 (csrc/arc_sim.c:26-54). n_worlds worlds of
 * the quadruped on flat grid x grid terrain; grid is clamped to 64.
 * Returns NULL if no CUDA device is usable or memory runs out. Steps in
 * FP32 with the warp-per-leg kernel (see arc_sim_create_ex). */
arc_sim *arc_sim_create(int n_worlds, double dt, int substeps, int grid, double cell);

/* Replaces csrc/arc_sim.h:26. NULL-safe. */
void arc_sim_destroy(arc_sim *s);

/* Replaces csrc/arc_sim.h:27: stored (<= 0 -> 1); the GPU ignores it. */
void arc_sim_set_threads(arc_sim *s, int threads);

/* Replace csrc/arc_sim.h:28-30. */
int arc_sim_num_worlds(const arc_sim *s);
int arc_sim_num_joints(void);
int arc_sim_num_legs(void);

/* Replaces csrc/arc_sim.h:33: default_angles, lo, hi are 12 doubles each,
 * misc = {stand height, total mass}; any pointer may be NULL. */
void arc_sim_robot_info(const arc_sim *s, double *default_angles, double *lo, double *hi, double *misc);

/* Replaces csrc/arc_sim.h:38: regenerates the listed worlds' terrain from
 * (seed, difficulty) and drops the robot in a noisy default stance with a
 * random yaw, exactly as the reference's RNG stream dictates. */
void arc_sim_reset(arc_sim *s, const int *ids, int n_ids, const unsigned int *seeds, const double *difficulty);

/* Replaces csrc/arc_sim.h:42: targets is N x 12 drive targets (rad),
 * clamped to the joint limits; unstable worlds are not stepped. */
void arc_sim_step(arc_sim *s, const double *targets);

/* Replaces csrc/arc_sim.h:46: root N x 13, rot N x 9, joints N x 36,
 * contacts N x 6, flags N; any pointer may be NULL. */
void arc_sim_observe(const arc_sim *s, double *root, double *rot, double *joints, double *contacts, int *flags);

/* Replaces csrc/arc_sim.h:51: heights at k (forward, left) offsets in each
 * torso's heading frame; out is N x k. */
void arc_sim_heights(const arc_sim *s, const double *offsets, int k, double *out);

/* Replaces csrc/arc_sim.h:54: height at point i (xy[2i], xy[2i+1]) of world ids[i]. */
void arc_sim_terrain_at(const arc_sim *s, const int *ids, const double *xy, int m, double *out);

/* Replaces csrc/arc_sim.h:56: a host FP64 copy of world i in the
 * reference's arc_world layout (arc_world.h), refreshed from the device by
 * this call and valid until the next arc_sim_world call on the same sim.
 * The robot's render-only visuals are filled in from the model (n_visuals
 * is the model's count). The contact list (n_contacts, contacts) is the last
 * substep's, in the reference's order, once the step kernels record it: the
 * first arc_sim_world call on a sim turns recording on (see
 * arc_sim_set_record_contacts), so it returns n_contacts = 0 and later calls
 * return the list of the latest step. */
const arc_world *arc_sim_world(const arc_sim *s, int i);

/* ======================================================================
 * Part 2: additive API (no counterpart in the reference)
 * ====================================================================== */

/* status codes */
#define ARC_OK 0
#define ARC_ERR_CUDA (-1)       /* a CUDA call failed; see arc_sim_error_message */
#define ARC_ERR_ARG (-2)        /* bad argument (index, size, pointer) */
#define ARC_ERR_UNSUPPORTED (-3) /* e.g. leg-parallel kernel on a non-quadruped model */

/* create flags */
#define ARC_SIM_FP64 1u         /* step in FP64 instead of FP32 */
#define ARC_SIM_PLAIN 2u        /* start with the plain per-world kernel */

/* kernels */
#define ARC_KERNEL_PLAIN 0      /* one thread per world */
#define ARC_KERNEL_LEGS 1       /* four lanes per world (one per leg), shared-memory staging */
#define ARC_KERNEL_WARPS 2      /* four warps per 32 worlds (one warp per leg), state in shared memory;
                                   FP32, and FP64 with two CTAs per SM and no substep tiles */

arc_sim *arc_sim_create_ex(int n_worlds, double dt, int substeps, int grid, double cell, unsigned flags);

/* Worlds whose terrain grids differ: world i holds grids[i] x grids[i]
 * columns (1..64), all packed in one pool, and arc_sim_reset generates a
 * grids[i]-sized terrain for it (the reference's arc_terrain takes nx, ny
 * per world, csrc/arc_terrain.h:13-20; its arc_sim has one grid for all,
 * csrc/arc_sim.c:36). arc_sim_set_terrain may then write at most
 * grids[i]^2 columns. NULL on a size outside 1..64 or no device. */
arc_sim *arc_sim_create_sized(int n_worlds, const int *grids, double dt, int substeps, double cell, unsigned flags);

/* Last error of any call on s (0 if none) and its message; clears nothing. */
int arc_sim_last_error(const arc_sim *s);
const char *arc_sim_error_message(const arc_sim *s);

/* Kernel choice; worlds_per_cta in {1, 2, 4, 8, 16, 32, 64} for
 * ARC_KERNEL_LEGS, four threads per world (ARC_KERNEL_WARPS always steps 32
 * worlds per CTA). */
int arc_sim_set_kernel(arc_sim *s, int kernel, int worlds_per_cta);
int arc_sim_get_kernel(const arc_sim *s, int *kernel, int *worlds_per_cta);
/* 4 for FP32, 8 for FP64 */
int arc_sim_real_size(const arc_sim *s);
/* Counts of the simulated model: bodies, joints, spheres, contact channels
 * (the quadruped: 13, 12, 21, 6); any pointer may be NULL. */
int arc_sim_model_info(const arc_sim *s, int *n_bodies, int *n_joints, int *n_spheres, int *n_channels);

/* World-state snapshots, host FP64 buffers of arc_sim_state_size doubles per
 * world: bodies (x3 q4 v3 w3) x nb, spheres (anchored, anchor3, anchor_n3,
 * touch) x ns, joints (target, angle, rate, torque) x nj, unstable, time. */
int arc_sim_state_size(const arc_sim *s);
int arc_sim_get_state(const arc_sim *s, const int *ids, int n_ids, double *out);
int arc_sim_set_state(arc_sim *s, const int *ids, int n_ids, const double *in);

/* Terrain of one world: nx x ny columns (heights[ix + iy * nx], FP64),
 * centred on the origin, `outside` beyond the grid; nx, ny <= the grid the
 * sim was created with. geom = {cell, ox, oy, outside}. */
int arc_sim_set_terrain(arc_sim *s, int id, int nx, int ny, double cell, double outside, const double *heights);
int arc_sim_get_terrain(const arc_sim *s, int id, int *nx_ny, double *geom, double *heights);

/* Gravity and friction coefficients of every world (csrc/arc_phys.c:32-39). */
int arc_sim_set_world_params(arc_sim *s, const double *gravity, double mu_static, double mu_dynamic);

/* Drive and limit parameters of joint j (lo > hi disables the limits). */
int arc_sim_set_joint(arc_sim *s, int j, double lo, double hi, double kp, double kd, double max_torque);

/* ---- custom models (csrc/arc_phys.h:114-144 builders), for scenes other
 * than the quadruped; they step with ARC_KERNEL_PLAIN. */
typedef struct arc_model arc_model;
arc_model *arc_model_create(void);
void arc_model_destroy(arc_model *m);
/* inertia: principal moments; q: w, x, y, z. Returns the index or -1. */
int arc_model_add_body(arc_model *m, double mass, const double *inertia, const double *pos, const double *q);
int arc_model_add_sphere(arc_model *m, int body, const double *local_pos, double radius);
int arc_model_add_hinge(arc_model *m, int parent, int child, const double *anchor, const double *axis);
/* A render-only visual in the body's frame (csrc/arc_phys.h:69-98): type
 * 0 sphere, 1 box, 2 taper, 3 cylinder, 4 ring; material 0 paint, 1 panels,
 * 2 metal, 3 rubber, 4 lens, 5 ribs, 6 glow; rgb in [0, 1]. Returns the
 * index or -1. */
int arc_model_add_visual(arc_model *m, int type, int body, const double *p0, const double *p1, double radius,
                         double radius2, double aspect, int material, const float *rgb);
arc_sim *arc_sim_create_model(const arc_model *m, int n_worlds, double dt, int substeps, int grid, double cell,
                              unsigned flags);
/* Places body 0 at (pos, q) and the others by forward kinematics from the
 * joint angles, zeroing velocities and setting drive targets to the angles
 * (csrc/arc_phys.c:749-782). */
int arc_sim_set_pose(arc_sim *s, int id, const double *pos, const double *q, const double *angles);

/* ---- device-resident path. Pointers are CUDA device pointers; stream is a
 * cudaStream_t (NULL: the sim's own stream). Calls are asynchronous on that
 * stream. */
void *arc_sim_stream(const arc_sim *s);
/* targets: N x 12 FP64 on the device */
int arc_sim_step_device(arc_sim *s, const double *d_targets, void *stream);
/* actions: N x 12 FP32 policy actions on the device; targets are
 * default + action_scale * clip(a, -1, 1) (arc/task.py:159-160), clamped */
int arc_sim_step_actions(arc_sim *s, const float *d_actions, void *stream);
/* observe into device FP64 buffers (any may be NULL) */
int arc_sim_observe_device(const arc_sim *s, double *root, double *rot, double *joints, double *contacts, int *flags,
                           void *stream);
int arc_sim_synchronize(const arc_sim *s);
/* Steps only the n_ids worlds d_ids[0..n_ids) (device ints, distinct; ids
 * outside 0..N-1 are skipped), with exactly one of d_targets (N x 12 FP64)
 * or d_actions (N x 12 FP32, as arc_sim_step_actions), read at the listed
 * rows only. Quadruped batches use the warp-per-leg kernel (FP32 or FP64)
 * unless the plain one is selected, other models the plain one. */
int arc_sim_step_ids(arc_sim *s, const int *d_ids, int n_ids, const double *d_targets, const float *d_actions,
                     void *stream);
/* observe of the listed worlds (device ids) into device buffers whose row k
 * belongs to world d_ids[k] (same blocks as arc_sim_observe; any may be NULL) */
int arc_sim_observe_ids(const arc_sim *s, const int *d_ids, int n_ids, double *root, double *rot, double *joints,
                        double *contacts, int *flags, void *stream);
/* on != 0: the warp-per-leg kernel runs one wave of resident CTAs that take
 * groups of 32 worlds from a device work queue, instead of one CTA per group */
int arc_sim_set_work_queue(arc_sim *s, int on);
/* Substep tiling of the FP32 warp-per-leg kernel: tile in 1 .. substeps - 1 runs
 * each control step as launches of `tile` substeps, the state going through
 * device memory between them (the same worlds bit for bit); 0 (the default)
 * or >= substeps: the whole control step in one launch, the state on chip
 * throughout. FP64 sims refuse tiles (ARC_ERR_UNSUPPORTED). */
int arc_sim_set_substep_tile(arc_sim *s, int tile);
/* on != 0: the step kernels keep each world's contact list of the last
 * substep on the device (128 records a world: 4 KB in FP32, 8 KB in FP64),
 * which arc_sim_world returns; 0 frees it. Off until set or until the first
 * arc_sim_world call. */
int arc_sim_set_record_contacts(arc_sim *s, int on);

/* The checked build (libarcsim_checked.so, compiled with ARC_DEVICE_CHECKS)
 * tests the kernels' data-dependent indexes - terrain columns against their
 * world's slice of the terrain pool, contact records against their lane's
 * slice of the spill buffer - and skips an access that fails, recording it.
 * This call reads the record of every kernel of the library: the number of
 * failed checks since the last clear, the site of the first (1 terrain read
 * in a step, 2/3 contact spill write/read, 4 observation height or terrain
 * lookup, 5 terrain write of a reset) and its index; clear != 0 zeroes the
 * record. Returns 1 for the checked build, 0 for the regular build (which
 * checks nothing and reports zeros), < 0 on a CUDA error. */
int arc_device_checks(unsigned long long *failures, int *first_site, long long *first_index, int clear);

/* Measured FP32 FMA throughput of the current device (FLOP/s, an FMA
 * counted as 2): the roofline denominator of the step kernels. */
int arc_probe_fp32_peak(double *flops_per_s, double *seconds);

/* ---- one control step without any device allocation. No counterpart in
 * the reference: for callers that cannot call cudaMalloc (a host runtime
 * that owns all device memory through its own arena; a control loop that
 * must not trigger cudaMalloc's device-wide synchronisation), which
 * therefore cannot create an arc_sim. The caller owns every buffer:
 *   d_state    n_worlds x arc_sim_state_size (387) FP64, the snapshot layout
 *              of arc_sim_get_state, read and updated in place
 *   d_heights  n_worlds x grid x grid FP32 column heights, h[ix + iy * grid],
 *              grid centred on the origin, `outside` beyond it
 *   d_targets  n_worlds x 12 FP64 drive targets (as arc_sim_step)
 * and the quadruped steps in FP32 with the leg-parallel kernel, asynchronously
 * on `stream`. The kernel's work memory is one static device array of the
 * library (about 4.9 MB, held by every GPU that loads the library until exit),
 * which limits a call to n_worlds <= 1024, grid <= 64, cell >= 0.4 m and
 * substeps <= 1023;
 * larger requests return ARC_ERR_ARG. The first call on a device looks up the
 * array's device address; make that first call before any stream capture.
 * That address is kept for the life of the process: after cudaDeviceReset on
 * a device the array moves, so a process that resets a device must not call
 * arc_step_noalloc on it again.
 * Every call shares the array, so calls whose work overlaps on the GPU race:
 * serialise them (one stream, or events). */
int arc_step_noalloc(double *d_state, const float *d_heights, int grid, double cell, double outside,
                     const double *d_targets, int n_worlds, double dt, int substeps, void *stream);

/* ---- the task layer on the device (arc/task.py ArcTask and the auto-reset
 * of arc/env.py ArcVecEnv.step_wait), so a training loop keeps observations,
 * rewards and done flags in device memory. */

/* TaskConfig (arc/task.py:17-66); arc_task_config_default fills its defaults. */
typedef struct arc_task_config {
    double dt;
    int max_steps;
    double action_scale, checkpoint_radius, checkpoint_min_dist, checkpoint_max_dist, border;
    double w_progress, max_speed, fov, w_turn, w_checkpoint, w_time, w_fall, w_energy, w_action_rate;
    double w_body_contact, w_torso_contact, w_body_rate, w_bounce;
    double flip_up_z;
    int beached_steps;
    double void_z;
    int curriculum;
    double difficulty, max_difficulty, level_step;
    int level_up_checkpoints, level_down_steps;
} arc_task_config;

void arc_task_config_default(arc_task_config *c);

/* Attaches task state and output buffers to s. seed starts the device
 * random stream of reset seeds and checkpoint draws (the reference draws
 * them from numpy's PCG64 on the host; the distributions are the same). */
int arc_env_init(arc_sim *s, const arc_task_config *cfg, unsigned long long seed);

/* ArcTask.reset (arc/task.py:113-125) of the listed worlds (host ids; NULL
 * and n_ids < 0: all), writing their observations. */
int arc_env_reset(arc_sim *s, const int *ids, int n_ids, void *stream);

/* One control step of ArcVecEnv.step_wait (arc/env.py:99-117) on the device:
 * actuation from d_actions (N x 12 float32, clipped to [-1, 1]), physics,
 * rewards, terminations, checkpoints, curriculum, observations, and the
 * reset of every world that ended (their pre-reset observation goes to
 * ARC_ENV_TERMINAL_OBS). d_actions == NULL: the ARC_ENV_ACTIONS buffer,
 * through a CUDA graph of the whole step captured on first use. With the
 * warp-per-leg kernel (FP32) the step and the task layer can run fused (see
 * arc_env_set_fused). */
int arc_env_step(arc_sim *s, const float *d_actions, void *stream);

/* Starts the listed worlds (host ids) afresh for a new tenant: difficulty
 * (level) per world, and a key per world that names its random streams
 * (reset seeds, checkpoints) in place of its index, with those streams
 * restarted; then ArcTask.reset and the observation. What such a world
 * draws depends on its key and not on which world slot it occupies, so a
 * tenant's worlds behave alike in any slots. Synchronous. */
int arc_env_admit(arc_sim *s, const int *ids, int n_ids, const double *difficulty, const unsigned *keys,
                  void *stream);

/* One control step of ArcVecEnv.step_wait for the listed worlds only
 * (device ids, distinct): their actions from the ARC_ENV_ACTIONS rows of
 * those worlds, their outputs in the env buffers' rows of those worlds, the
 * ended ones (ARC_ENV_DONE_LIST / DONE_COUNT) reset. Asynchronous on stream. */
int arc_env_step_ids(arc_sim *s, const int *d_ids, int n_ids, void *stream);

/* How the env's control step (arc_env_step, arc_env_step_part,
 * arc_env_step_host, arc_env_step_ids) runs with the warp-per-leg kernel:
 * 0 (the default) the step kernel, then the task, heights and reset kernels;
 * 1 each group of 32 worlds stepped and then given its rewards,
 * observations and heights in the same kernel, the ended worlds reset by the
 * reset kernel after it; 2 the ended worlds reset in that kernel too (one
 * launch per control step). The task layer's results are the same in all
 * three; the physics of forms 1 and 2 is compiled into their own kernel and
 * agrees with form 0's to FP32 rounding (form 0, the fastest, keeps the
 * task code out of the step kernel). */
int arc_env_set_fused(arc_sim *s, int mode);

/* The order in which the env's control step hands worlds to the step
 * kernels (warp-per-leg and plain): 1 (the default) the worlds of each
 * range stepped (all worlds, a part of arc_env_step_part, a chunk of
 * arc_env_step_host) by difficulty band (16 bands, hardest first; by index
 * within a band), made from the current difficulties every step, so that
 * the costliest groups of 32 worlds go first and the cheapest run while the
 * GPU empties; 0 index order. A world's results do not depend on the order:
 * both modes give the same worlds bit for bit. */
int arc_env_set_step_order(arc_sim *s, int mode);

/* The order (N world indices, a permutation) that a whole control step
 * hands the step kernels now; synchronous. */
int arc_env_get_step_order(arc_sim *s, int *order);

/*
 * The same control step with host buffers, as ArcVecEnv.step_wait's caller
 * sees it (arc/env.py:99-117): h_actions (N x 12 float32) in; observations
 * (N x 195 float32), rewards (N float32), terminated and truncated (N
 * bytes) out; any output but the observations may be NULL. The worlds are
 * stepped in `chunks` contiguous ranges (1..16), each about half the size
 * of the one before, so that the copies of one range overlap the step of
 * the next: with page-locked host buffers only the last, smallest range's
 * copies add to the step's time. Results equal
 * arc_env_step's followed by copies, world for world (with the leg-parallel
 * kernel selected, ranges step on the warp-per-leg kernel, which agrees with
 * it to FP32 rounding rather than bit for bit); the ended-world list
 * (ARC_ENV_DONE_LIST / DONE_COUNT) is filled in range order. Runs after the
 * work queued on the sim's own stream; work the caller queued on other
 * streams (e.g. arc_env_step on its own stream) must have finished.
 * Synchronous: returns when the host buffers hold the results.
 */
int arc_env_step_host(arc_sim *s, const float *h_actions, float *h_obs, float *h_reward, unsigned char *h_terminated,
                      unsigned char *h_truncated, int chunks);

/*
 * The control step of arc_env_step in `parts` contiguous ranges of
 * near-equal size (1..16 parts, at most one per world), each stepped
 * into the caller's stream: part `part` covers worlds first .. first +
 * count - 1 (arc_env_part_range). Parts may run at the same time on
 * different streams (each has its own work queue and ended-world list), so
 * that a policy evaluated on one part's observations overlaps the step of
 * another, which fills the step kernel's last, partly filled wave of
 * blocks. Each part reads its rows of the ARC_ENV_ACTIONS buffer and writes
 * its rows of every output; world for world the results equal
 * arc_env_step's (the same caveat for the leg-parallel kernel as
 * arc_env_step_host's). Once every part of a step has been queued,
 * arc_env_merge_parts (on a stream that waited for all parts) fills
 * ARC_ENV_DONE_LIST / DONE_COUNT in part order. No arc_env_step_host or
 * second set of parts may run while parts are in flight.
 */
int arc_env_part_range(const arc_sim *s, int part, int parts, int *first, int *count);
int arc_env_step_part(arc_sim *s, int part, int parts, void *stream);
int arc_env_merge_parts(arc_sim *s, int parts, void *stream);

/* ArcTask.step alone (arc/task.py:155-220): no observation, no reset. */
int arc_env_task_step(arc_sim *s, const float *d_actions, void *stream);
/* ArcTask.observe (arc/task.py:231-259) of every world into ARC_ENV_OBS. */
int arc_env_observe(arc_sim *s, void *stream);

/* device buffers of the task layer */
#define ARC_ENV_OBS 0               /* float32 N x 195 */
#define ARC_ENV_TERMINAL_OBS 1      /* float32 N x 195 (rows of worlds that ended) */
#define ARC_ENV_REWARD 2            /* float32 N */
#define ARC_ENV_TERMINATED 3        /* uint8 N */
#define ARC_ENV_TRUNCATED 4         /* uint8 N */
#define ARC_ENV_CAUSE 5             /* int8 N: "", unstable, void, flip, beached */
#define ARC_ENV_DONE_LIST 6         /* int32 N: worlds that ended in the last step */
#define ARC_ENV_DONE_COUNT 7        /* int32 1 */
#define ARC_ENV_ACTIONS 8           /* float32 N x 12: input of arc_env_step(s, NULL, ...) */
#define ARC_ENV_ENDED_CHECKPOINTS 9 /* int32 N: episode stats of worlds that ended */
#define ARC_ENV_ENDED_STEPS 10      /* int32 N */
#define ARC_ENV_ENDED_DIFFICULTY 11 /* float64 N */
#define ARC_ENV_NUM_BUFFERS 12

/* Device pointer, shape (up to 2 dims) and dtype (DLPack codes: 0 int,
 * 1 uint, 2 float; bits) of a buffer. */
int arc_env_buffer(const arc_sim *s, int which, void **ptr, long long *shape, int *ndim, int *dtype_code,
                   int *dtype_bits);
/* Synchronous copies between a task-layer buffer and host memory of the
 * buffer's full size (the reference's host-buffer style). */
int arc_env_download(const arc_sim *s, int which, void *host);
int arc_env_upload(arc_sim *s, int which, const void *host);
/* The same buffer as a DLPack DLManagedTensor (caller hands it to a DLPack
 * consumer, which calls its deleter). The memory stays owned by s. */
int arc_env_dlpack(const arc_sim *s, int which, void **managed);

/* Per-world task state, host FP64, ARC_TASK_STATE_SIZE values per world:
 * target x y, target_z, prev_dist, prev_gaze, prev_action x12, torso_steps,
 * steps, checkpoints, level, difficulty, in_view, episode, draws. */
#define ARC_TASK_STATE_SIZE 25
int arc_env_get_task_state(const arc_sim *s, const int *ids, int n_ids, double *out);
int arc_env_set_task_state(arc_sim *s, const int *ids, int n_ids, const double *in);
/* Places checkpoints at given points (target_z, prev_dist, prev_gaze follow). */
int arc_env_set_targets(arc_sim *s, const int *ids, int n_ids, const double *xy);

/* ---- serving engine. No counterpart in the reference, which steps one
 * synchronous batch per call. A fixed pool of `capacity` world slots (the
 * device-memory budget) with the task layer, and one engine thread doing
 * continuous batching for any number of client threads:
 *   - a session is one client's batch of worlds. It waits for free slots,
 *     then is admitted: each world starts an episode at the session's
 *     difficulty (its random streams named by the session's key, so the
 *     same session gives the same worlds whichever slots it gets). Its worlds
 *     stay resident, episode after episode, until the session is closed.
 *   - a request steps one session's worlds n_steps control steps with the
 *     task layer; a world whose episode ends is evicted from its slot and the
 *     slot reset with its next episode at once (ArcVecEnv's auto-reset,
 *     arc/env.py:99-117), and the request goes on.
 *   - each tick steps the worlds of every running request in one launch. A
 *     queued request starts running, first come first served, when its
 *     session is resident and idle and the tick holds at most tick_cap
 *     worlds with it (a request larger than tick_cap runs alone).
 * A session's results in the mix equal its results alone, bit for bit. */
typedef struct arc_server arc_server;
/* dt, substeps, grid, cell as arc_sim_create; cfg the task (NULL: the
 * defaults with the curriculum off, so worlds keep their session's
 * difficulty); tick_cap 0: capacity. NULL on failure. */
arc_server *arc_server_create(int capacity, double dt, int substeps, int grid, double cell,
                              const arc_task_config *cfg, int tick_cap);
/* Stops the engine; queued requests fail. */
void arc_server_destroy(arc_server *sv);
/* A session of n_worlds worlds at difficulty[i] (copied), random streams
 * named by key. Returns its id (> 0) or < 0. */
long long arc_server_open(arc_server *sv, int n_worlds, const double *difficulty, unsigned long long key);
/* A request on a session: n_steps control steps with actions (n_steps x
 * n_worlds x 12 float32 in [-1, 1], copied) or, with actions NULL, an
 * Ornstein-Uhlenbeck process per world (theta 0.15, sigma 0.3, clipped to
 * [-1, 1]) seeded by ou_seed. Results into the caller's buffers, kept alive
 * until the wait returns (any may be NULL): obs n_worlds x 195 float32 after
 * the last step, reward n_steps x n_worlds float32, done n_steps x n_worlds
 * (bit 0 terminated, bit 1 truncated; the world was reset after that step).
 * A session's requests run one after another in submission order. Returns
 * the request id (> 0) or < 0. */
long long arc_server_request(arc_server *sv, long long session, int n_steps, const float *actions,
                             unsigned long long ou_seed, float *obs, float *reward, unsigned char *done);
/* Waits up to timeout_s for a request: 1 done (times: seconds queued,
 * running, total; may be NULL), 0 on timeout, < 0 on error. An id is
 * returned once. */
int arc_server_wait(arc_server *sv, long long request, double timeout_s, double *times);
/* Closes a session: its slots are freed once its submitted requests are
 * done; later requests on it fail. */
int arc_server_close(arc_server *sv, long long session);
/* stats (12 doubles): ticks, world-steps, engine busy seconds, most worlds
 * in one tick, completed requests, queued requests, busy seconds in
 * admission, stepping and reading results back, episodes ended, resident
 * worlds, sessions waiting for slots. Returns the engine's error (0 ok). */
int arc_server_stats(arc_server *sv, double *stats);

#ifdef __cplusplus
}
#endif

#endif
