// arc_step_plain.cu - the plain per-world step kernel.
//
// One thread steps one world: it copies the world's record from HBM into
// thread-local arrays, runs arc_world_step (csrc/arc_phys.c:707-747) on them
// and writes the record back. Any model up to the reference's capacities
// (16 bodies, 16 joints, 48 spheres, 128 contacts) runs here, so this kernel
// also carries the analytic known-answer scenes (free fall, pendulum, chain,
// ...). It is the baseline that the leg-parallel kernel is measured against.
#include "arc_kernels.cuh"

namespace arc {

template <class R>
__global__ void __launch_bounds__(128)
k_step_plain(const __grid_constant__ DevModel<R> M, Worlds<R> W, Actuation A, const int* __restrict__ ids,
             int n_ids)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_ids)
        return;
    const int i = ids ? ids[k] : k;
    if (i < 0 || i >= W.n)
        return;
    R* rec = W.rec + (size_t)i * W.stride;
    R* jr = rec + W.off_joint;
    R* sr = rec + W.off_sphere;
    uint32_t* sph = W.sph + (size_t)i * M.ns;
    const int nb = M.nb, nj = M.nj, ns = M.ns;

    // actuation (csrc/arc_sim.c:132-136)
    for (int j = 0; j < nj; ++j)
        jr[j * kJointRec] = actuate(M, A, i, j);
    if (W.unstable[i])
        return;

    Pose<R> P[kMaxBodies];
    V3<R> V[kMaxBodies], Wv[kMaxBodies], XP[kMaxBodies];
    Q4<R> QP[kMaxBodies];
    SphereState<R> S[kMaxSpheres];
    int touch[kMaxSpheres];
    R target[kMaxJoints], tacc[kMaxJoints];
    ContactRec<R> C[kMaxContacts];
    int CB[kMaxContacts];

    for (int b = 0; b < nb; ++b) {
        const R* r = rec + b * kBodyRec;
        P[b].x = V3<R>{r[0], r[1], r[2]};
        P[b].q = Q4<R>{r[3], r[4], r[5], r[6]};
        V[b] = V3<R>{r[7], r[8], r[9]};
        Wv[b] = V3<R>{r[10], r[11], r[12]};
        body_sync(P[b], M.body[b]);
    }
    for (int s = 0; s < ns; ++s) {
        const R* r = sr + s * kSphereRec;
        S[s].anchor = V3<R>{r[0], r[1], r[2]};
        S[s].anchor_n = V3<R>{r[3], r[4], r[5]};
        S[s].anchored = (sph[s] >> 16) & 1;
        touch[s] = 0;
    }
    for (int j = 0; j < nj; ++j) {
        target[j] = jr[j * kJointRec];
        tacc[j] = R(0);
    }
    const TerrainView<R> T = terrain_of(W, i);
    const StepK<R>& st = M.step;

    for (int sub = 0; sub < M.substeps; ++sub) {
        for (int b = 0; b < nb; ++b)
            integrate_body(P[b], V[b], Wv[b], XP[b], QP[b], M.body[b], st);
        int nc = 0;
        for (int j = 0; j < nj; ++j) {
            const JointK<R>& jk = M.joint[j];
            JointStepK<R> js = joint_step_k(jk, st);
            const int c = jk.child;
            if (jk.parent >= 0) {
                const int p = jk.parent;
                joint_positions<R, true>(P[p], M.body[p], P[c], M.body[c], jk, js, target[j], tacc[j], st.hh);
            } else {
                joint_positions<R, false>(P[c], M.body[c], P[c], M.body[c], jk, js, target[j], tacc[j], st.hh);
            }
        }
        for (int s = 0; s < ns; ++s) {
            const SphereK<R>& sk = M.sphere[s];
            const int b = sk.body;
            touch[s] += collide_sphere(P[b], M.body[b], XP[b], QP[b], sk, S[s], T, st,
                                       [&](V3<R> local, V3<R> n) {
                                           if (nc < kMaxContacts) {
                                               C[nc] = ContactRec<R>{local, n};
                                               CB[nc] = b;
                                               ++nc;
                                           }
                                       });
        }
        for (int b = 0; b < nb; ++b)
            update_velocity(P[b].q, P[b].x, V[b], Wv[b], XP[b], QP[b], st);
        for (int j = 0; j < nj; ++j) {
            const JointK<R>& jk = M.joint[j];
            JointStepK<R> js = joint_step_k(jk, st);
            const int c = jk.child;
            if (jk.parent >= 0) {
                const int p = jk.parent;
                joint_velocities<R, true>(P[p].rot, P[p].iiw, Wv[p], P[c].iiw, Wv[c], jk, js, st.h, tacc[j]);
            } else {
                V3<R> dummy{R(0), R(0), R(0)};
                joint_velocities<R, false>(P[c].rot, P[c].iiw, dummy, P[c].iiw, Wv[c], jk, js, st.h, tacc[j]);
            }
        }
        for (int c = 0; c < nc; ++c) {
            const int b = CB[c];
            contact_velocity(P[b].rot, P[b].iiw, M.body[b].inv_mass, V[b], Wv[b], C[c]);
        }
        if (W.lastc && sub == M.substeps - 1) {
            // the list the reference leaves in its world after a step
            R* d = W.lastc + (size_t)i * kMaxContacts * kContactRec;
            for (int c = 0; c < nc; ++c, d += kContactRec) {
                d[0] = (R)CB[c];
                d[1] = C[c].local.x; d[2] = C[c].local.y; d[3] = C[c].local.z;
                d[4] = C[c].n.x; d[5] = C[c].n.y; d[6] = C[c].n.z;
            }
            W.lastn[i] = nc;
        }
    }

    // epilogue (csrc/arc_phys.c:739-746)
    for (int j = 0; j < nj; ++j) {
        const JointK<R>& jk = M.joint[j];
        Q4<R> qp = jk.parent >= 0 ? P[jk.parent].q : q_identity<R>();
        V3<R> wp = jk.parent >= 0 ? Wv[jk.parent] : V3<R>{R(0), R(0), R(0)};
        R* o = jr + j * kJointRec;
        o[1] = joint_angle(qp, P[jk.child].q, jk);
        o[2] = joint_rate(qp, wp, Wv[jk.child], jk);
        o[3] = tacc[j] / R(M.substeps);
    }
    bool bad = false;
    for (int b = 0; b < nb; ++b) {
        bad |= body_unstable(P[b].x, V[b], Wv[b]);
        R* r = rec + b * kBodyRec;
        r[0] = P[b].x.x; r[1] = P[b].x.y; r[2] = P[b].x.z;
        r[3] = P[b].q.w; r[4] = P[b].q.x; r[5] = P[b].q.y; r[6] = P[b].q.z;
        r[7] = V[b].x; r[8] = V[b].y; r[9] = V[b].z;
        r[10] = Wv[b].x; r[11] = Wv[b].y; r[12] = Wv[b].z;
    }
    for (int s = 0; s < ns; ++s) {
        R* r = sr + s * kSphereRec;
        r[0] = S[s].anchor.x; r[1] = S[s].anchor.y; r[2] = S[s].anchor.z;
        r[3] = S[s].anchor_n.x; r[4] = S[s].anchor_n.y; r[5] = S[s].anchor_n.z;
        sph[s] = (uint32_t)touch[s] | ((uint32_t)(S[s].anchored != 0) << 16);
    }
    W.time[i] += M.step_dt;
    if (bad)
        W.unstable[i] = 1;
}

template <class R>
cudaError_t launch_step_plain(const DevModel<R>& M, const Worlds<R>& W, const Actuation& A, const int* ids,
                              int n_ids, cudaStream_t stream)
{
    if (n_ids <= 0)
        return cudaSuccess;
    const int threads = 128;
    k_step_plain<R><<<(n_ids + threads - 1) / threads, threads, 0, stream>>>(M, W, A, ids, n_ids);
    return cudaGetLastError();
}

template cudaError_t launch_step_plain<float>(const DevModel<float>&, const Worlds<float>&, const Actuation&,
                                              const int*, int, cudaStream_t);
template cudaError_t launch_step_plain<double>(const DevModel<double>&, const Worlds<double>&, const Actuation&,
                                               const int*, int, cudaStream_t);

}  // namespace arc
