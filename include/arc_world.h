/*
 * arc_world.h - host FP64 world record returned by arc_sim_world.
 *
 * Binary layout: the same field order, types and capacities as the
 * reference's arc_world (csrc/arc_phys.h:25-112, csrc/arc_terrain.h:13-19,
 * 62,960 bytes), so code compiled against the reference's headers reads the
 * record this library returns. The type names here are this library's own.
 */
#ifndef ARC_WORLD_H
#define ARC_WORLD_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double x, y, z; } arcw_vec3;
typedef struct { double w, x, y, z; } arcw_quat;
typedef struct { double m[3][3]; } arcw_mat3;

typedef struct {
    arcw_vec3 x, x_prev;
    arcw_quat q, q_prev;
    arcw_vec3 v, w;
    double mass, inv_mass;
    arcw_vec3 inertia, inv_inertia;
    arcw_mat3 rot, inv_iw;
} arcw_body;

typedef struct {
    int body;
    arcw_vec3 pos;
    double radius;
    int touch, anchored;
    arcw_vec3 anchor, anchor_n;
} arcw_sphere;

typedef struct {
    int parent, child;
    arcw_vec3 r1, r2, a1, a2, b1, b2;
    arcw_quat q_rel0;
    double lo, hi, kp, kd, max_torque, target;
    double angle, rate, torque, torque_acc;
    double lim[4];
} arcw_joint;

typedef struct {
    int body;
    arcw_vec3 local, n;
} arcw_contact;

typedef struct {
    int type, body;
    arcw_vec3 p0, p1;
    double radius, radius2, aspect;
    int material;
    float color[3];
} arcw_visual;

typedef struct {
    int nx, ny;
    double cell, ox, oy, outside;
    double h[64 * 64];
} arcw_terrain;

typedef struct arc_world {
    arcw_vec3 gravity;
    double mu_static, mu_dynamic;
    int n_bodies, n_joints, n_spheres, n_contacts, n_visuals;
    int unstable;
    double time;
    arcw_body bodies[16];
    arcw_joint joints[16];
    arcw_sphere spheres[48];
    arcw_contact contacts[128];
    arcw_visual visuals[80];
    arcw_terrain terrain;
} arc_world;

#ifdef __cplusplus
}
#endif

#endif
