/*
 * arc_render.h - headless renderer of the worlds of an arc_sim into RGB
 * frames, on the GPU.
 *
 * The first block is the reference's renderer ABI (csrc/arc_render.h:11-39,
 * bound by arc/native.py:59-70 from libarcrender.so): the same names,
 * arguments and meaning, drawing one world per call into a host buffer.
 * There is no window system: a visible renderer cannot be created (create
 * returns NULL, as the reference does without a display), the key list is
 * always empty and titles are ignored. The scene, the look and the camera
 * follow csrc/arc_render.c; the picture is ray cast on the GPU rather than
 * rasterised by OpenGL.
 *
 * The second block renders many worlds in one launch into device memory,
 * one camera per world.
 */
#ifndef ARC_RENDER_H
#define ARC_RENDER_H

#include "arc_sim.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct arc_renderer arc_renderer;

/* ---- the reference ABI (csrc/arc_render.h) */

/* Frames of width x height pixels. visible != 0 asks for a window, which
 * this renderer does not have: it returns NULL. Also NULL on a bad size
 * or when CUDA fails. */
arc_renderer *arc_render_create(int width, int height, int visible);
void arc_render_destroy(arc_renderer *r);

/*
 * Draws world `world` of the simulation. markers: n_markers checkpoints as
 * (x, y, z, radius), the one at index `active` highlighted (-1: none).
 * If rgb is not NULL, it receives width * height * 3 bytes, top row first.
 * Returns 1, or 0 on an error (bad world index, CUDA failure); it never
 * reports a closed window because there is none.
 */
int arc_render_frame(arc_renderer *r, const arc_sim *s, int world, const double *markers, int n_markers, int active,
                     unsigned char *rgb);

void arc_render_size(const arc_renderer *r, int *width, int *height);

/* No window, no keys: always 0. */
int arc_render_keys(arc_renderer *r, int *keys, int max);

/* No window: ignored. */
void arc_render_set_title(arc_renderer *r, const char *title);

/* Camera presets around the robot's heading: 0 behind, 1 side, 2 front
 * (any integer, taken modulo 3). */
void arc_render_set_view(arc_renderer *r, int preset);

/* ---- batched device rendering */

/* Rays per pixel: 1 (pixel centres) or 4 (the default; the sample pattern
 * of 4x multisampling, which the reference's offscreen frames use). */
int arc_render_set_samples(arc_renderer *r, int samples);

/* Forgets every camera: the next frame of each world starts behind its
 * robot, without smoothing. */
int arc_render_reset_cameras(arc_renderer *r);

/*
 * Renders the n distinct worlds d_ids[0..n) of s (d_ids NULL: worlds 0..n-1) into
 * d_rgb, n x height x width x 3 bytes on the device, top rows first.
 * d_markers: NULL, or n x markers_per_world x 4 floats (x, y, z, radius)
 * on the device; d_active: NULL (none highlighted) or n ints, the
 * highlighted marker of each world or -1. markers_per_world <= 4. Each
 * world has its own camera, which follows its robot from frame to frame
 * like the reference's single camera. Asynchronous on `stream` (NULL: the
 * sim's stream); a call on another stream than the previous call's waits
 * for it. Returns ARC_OK or an ARC_ERR_* code.
 */
int arc_render_frames(arc_renderer *r, const arc_sim *s, const int *d_ids, int n, const float *d_markers,
                      int markers_per_world, const int *d_active, unsigned char *d_rgb, void *stream);

/*
 * The worlds of a sim whose device task layer is initialised (arc_env_init)
 * rendered like arc_render_frames, each with its current checkpoint as the
 * marker, highlighted while the robot sees it (arc/env.py:45-47,
 * arc/task.py:261-264). ARC_ERR_ARG without a task layer.
 */
int arc_env_render(arc_renderer *r, const arc_sim *s, const int *d_ids, int n, unsigned char *d_rgb, void *stream);

#ifdef __cplusplus
}
#endif

#endif
