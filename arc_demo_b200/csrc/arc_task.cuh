// arc_task.cuh - the task layer on the device: observations, rewards,
// terminations, checkpoints and the terrain curriculum of the reference's
// arc/task.py (ArcTask), computed in FP64 from the step-precision state.
#pragma once

#include "arc_kernels.cuh"

struct arc_sim;

namespace arc {

constexpr int kNumOffsets = 143;                 // arc/task.py:74-76: 13 forward x 11 left
constexpr int kObsSize = 9 + 3 * kNumJoints + 3 + kNumOffsets + kNumLegs;  // 195

// TaskConfig (arc/task.py:17-66) plus derived constants.
struct TaskParams {
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
    // derived
    double cos_fov, fov_rad, half_extent, stand_height;
    double default_angles[kNumJoints];
    double offsets[kNumOffsets][2];
    unsigned long long seed;  // device RNG stream of resets and checkpoint draws
};

// Per-world task state (the ArcTask arrays, arc/task.py:96-109), device arrays.
struct TaskState {
    double* target;       // [N][2]
    double* target_z;     // [N]
    double* prev_dist;    // [N]
    double* prev_gaze;    // [N]
    float* prev_action;   // [N][12] (clipped float32 actions: exact in float)
    int* torso_steps;     // [N]
    int* steps;           // [N]
    int* checkpoints;     // [N]
    double* level;        // [N]
    double* difficulty;   // [N]
    unsigned char* in_view;  // [N]
    unsigned* episode;    // [N] resets so far (device RNG counter)
    unsigned* draws;      // [N] checkpoint draws so far (device RNG counter)
    unsigned* key;        // [N] identity of each world's RNG streams (NULL: the world index)
};

// Outputs of one env step, device arrays.
struct TaskOut {
    float* obs;            // [N][195]
    float* terminal_obs;   // [N][195], rows of worlds that ended this step
    float* reward;         // [N]
    unsigned char* terminated, *truncated;  // [N]
    signed char* cause;    // [N] index into ("", unstable, void, flip, beached)
    int* ended_checkpoints;   // [N] episode stats of worlds that ended this step
    double* ended_difficulty; // [N]
    int* ended_steps;         // [N]
    int* done_list;        // [N] worlds that ended this step
    int* done_count;       // [1]
};

template <class R>
// Worlds first .. first + count - 1 (count < 0: to the last world), or with
// ids the count worlds ids[0 .. count) (device array).
// write_obs: 0 no observation rows, 1 whole rows, 2 rows without the terrain
// heights, which launch_task_heights then writes with more threads.
cudaError_t launch_task_step(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskState& S,
                             const TaskOut& O, const float* actions, int write_obs, cudaStream_t stream, int first = 0,
                             int count = -1, const int* ids = nullptr);

template <class R>
cudaError_t launch_task_heights(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskOut& O,
                                cudaStream_t stream, int first = 0, int count = -1, const int* ids = nullptr);

template <class R>
cudaError_t launch_task_observe(const DevModel<R>& M, const Worlds<R>& W, const TaskParams& P, const TaskState& S,
                                float* obs, const int* ids, int n_ids, cudaStream_t stream);

// Task reset of worlds (arc/task.py:113-125): device-drawn seeds, terrain,
// pose, task state, a checkpoint, and their observations. ids == nullptr
// with count_dev != nullptr: the worlds listed in done_list[0..*count_dev).
template <class R>
cudaError_t launch_task_reset(const DevModel<R>& M, const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg,
                              TerrainGeomD* tgd, const int* grid_of, double cell, const TaskParams& P,
                              const TaskState& S, float* obs, const int* ids, const int* count_dev, int max_n,
                              cudaStream_t stream);

// The control step (step, rewards, terminations, observations and, with
// resets, the reset of ended worlds) fused into one launch, for the
// quadruped in FP32: the warp-per-leg step of each group of 32 worlds
// followed by the task layer on them. The worlds are ids[0 .. n_items) (ids
// nullptr: 0 .. n_items - 1); with a queue (two device ints, zero between
// launches) one wave of resident CTAs takes the groups. O.done_count must be
// zero before the launch. Without resets the ended worlds are only listed
// (O.done_list), for launch_task_reset. The results equal launch_step_warps,
// launch_task_step (write_obs 2), launch_task_heights and launch_task_reset
// over O.done_list in turn to FP32 rounding: the task functions are compiled
// once, and the physics is the same source compiled into this form's kernel.
cudaError_t launch_control_step(const DevModel<float>& M, const ResetModel& RM, const Worlds<float>& W,
                                TerrainGeom<float>* tg, TerrainGeomD* tgd, const int* grid_of, double cell,
                                const TaskParams& P, const TaskState& S, const TaskOut& O, const float* actions,
                                float* spill, int spill_per_lane, int lane_cap, const int* ids, int n_items, int* queue,
                                bool resets, cudaStream_t stream);

// Starts worlds ids[0 .. n) (device arrays) afresh as new tenants of their
// slots: level and difficulty, RNG key and RNG counters set, then a task
// reset (terrain, pose, task state, checkpoint, observation), so that what a
// world draws depends on its key, not on its slot. S.key must be allocated.
template <class R>
cudaError_t launch_env_admit(const DevModel<R>& M, const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg,
                             TerrainGeomD* tgd, const int* grid_of, double cell, const TaskParams& P,
                             const TaskState& S, float* obs, const int* ids, const double* difficulty,
                             const unsigned* keys, int n, cudaStream_t stream);

// Checkpoints at given points (host-injected; parity tests and callers that
// draw their own): target, target_z, prev_dist, prev_gaze, in_view.
template <class R>
cudaError_t launch_task_set_targets(const Worlds<R>& W, const TaskParams& P, const TaskState& S, const int* ids,
                                    const double* xy, int n, cudaStream_t stream);

// Warp-cooperative reset used by arc_sim_reset: seeds and difficulties given.
template <class R>
cudaError_t launch_reset_warp(const ResetModel& RM, const Worlds<R>& W, TerrainGeom<R>* tg, TerrainGeomD* tgd,
                              const int* ids, int n_ids, const unsigned* seeds, const double* difficulty,
                              const int* grid_of, double cell, cudaStream_t stream);

// The device task state of an arc_sim whose task layer is initialised
// (false otherwise), and its checkpoint radius; arc_sim.cu owns the struct.
bool sim_task_view(const arc_sim* s, TaskState* state, double* checkpoint_radius);

}  // namespace arc
