// arc_model.h - the robot template in FP64 on the host, and its device copies.
//
// The template is what csrc/arc_robot.c builds with csrc/arc_phys.c's
// builders: 13 bodies, 12 hinges with limits and PD drives, 21 collision
// spheres. It is computed once in FP64 (the reference's arithmetic) and
// rounded once into the step precision.
#pragma once

#include "arc_kernels.cuh"

struct arc_sim;

namespace arc {

// render-only visuals: shapes and surface looks of csrc/arc_phys.h:69-87
constexpr int kMaxVisuals = 80;
enum VisualType { kVisSphere = 0, kVisBox, kVisTaper, kVisCylinder, kVisRing };
enum Material { kMatPaint = 0, kMatPanels, kMatMetal, kMatRubber, kMatLens, kMatRibs, kMatGlow };

struct ModelHost {
    int nb = 0, nj = 0, ns = 0;
    V3<double> gravity{0.0, 0.0, -9.81};
    double mu_s = 1.0, mu_d = 0.8;  // csrc/arc_phys.c:32-39
    struct Body {
        double mass, inv_mass;
        V3<double> inertia, inv_inertia, x;
        Q4<double> q;
    } b[kMaxBodies];
    struct Joint {
        int parent, child;
        V3<double> r1, r2, a1, a2, b1, b2;
        Q4<double> q_rel0;
        double lo, hi, kp, kd, max_torque;
    } j[kMaxJoints];
    struct Sphere {
        int body;
        V3<double> pos;
        double radius;
    } s[kMaxSpheres];
    // render-only geometry in the body frame (csrc/arc_phys.h:69-98); the
    // solver never reads it
    struct Visual {
        int type, body, material;
        V3<double> p0, p1;
        double radius, radius2, aspect;
        float color[3];
    } v[kMaxVisuals];
    int nv = 0;
    int channel[kMaxSpheres] = {};
    int n_channels = 6;
    // robot info (csrc/arc_robot.h:22-30)
    int foot_sphere[kNumLegs] = {};
    int n_torso_spheres = 0;
    double default_angles[kMaxJoints] = {};
    double stand_height = 0.0, total_mass = 0.0, footprint = 0.0;
    bool leaper = false;

    // builders (csrc/arc_phys.c:84-143); return the new index or -1
    int add_body(double mass, V3<double> inertia, V3<double> pos, Q4<double> q);
    int add_sphere(int body, V3<double> pos, double radius);
    int add_hinge(int parent, int child, V3<double> anchor_world, V3<double> axis_world);
    // aspect 1; returns the new index or -1 (csrc/arc_phys.c:145-164)
    int add_visual(int type, int body, V3<double> p0, V3<double> p1, double radius, double radius2, int material,
                   const float* rgb);
    // forward kinematics of every body from the root pose and joint angles
    void pose(V3<double> root_x, Q4<double> root_q, const double* angles, V3<double>* xs,
              Q4<double>* qs) const;
};

// csrc/arc_robot.c:145-195
void build_leaper(ModelHost& m);

// true if the model has the leaper's topology, which the leg-parallel
// kernel is specialised for: body 0 the torso, joint 3k+c (c = 0, 1, 2) the
// chain torso -> coxa -> femur -> tibia of leg k, spheres on the torso,
// femurs and tibias only.
bool is_leaper_topology(const ModelHost& m);

// Upper bound of the contact records one lane of the leg-parallel kernel
// (one leg: its five spheres, and the torso's for leg 0) can make in one
// substep on columns of the given cell size (0 for other topologies).
int lane_contact_bound(const ModelHost& m, double cell);

// What the renderer reads of an arc_sim (arc_sim.cu owns the struct).
struct SimView {
    const ModelHost* model;
    Worlds<float> wf;
    Worlds<double> wd;
    bool fp64;
    int n;
    cudaStream_t stream;
};
SimView sim_view(const arc_sim* s);

template <class R> DevModel<R> make_dev_model(const ModelHost& m, double dt, int substeps, double action_scale);
ResetModel make_reset_model(const ModelHost& m);

V3<double> inertia_sphere(double mass, double r);
V3<double> inertia_box(double mass, V3<double> half_extents);
V3<double> inertia_capsule_z(double mass, double radius, double half_length);

}  // namespace arc
