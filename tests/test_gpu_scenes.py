"""The reference's analytic physics scenes (csrc/tests/test_phys.c and the
void scene of csrc/tests/test_robot.c) run through the CUDA library's
custom-model entry points, with the reference's own tolerances.

These pin the solver against closed-form answers (free fall, pendulum
period, gravity sag, stopping distance, ...), independent of any oracle.
FP64 runs use the reference's tolerances as they are; FP32 runs of the
same scenes use the tolerance noted beside each check where FP32 rounding
dominates (e.g. 1e-9 m position bounds become 1e-4 m).
"""

import numpy as np
import pytest

from arc_demo_b200.native import Model, Sim

pytestmark = pytest.mark.gpu

DT, SUB = 1.0 / 30.0, 20


def qaxis(axis, angle):
    axis = np.asarray(axis, dtype=float)
    return np.array([np.cos(0.5 * angle), *(axis * np.sin(0.5 * angle))])


def qrot(q, v):
    w, u = q[0], np.asarray(q[1:])
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def qinv(q):
    return np.array([q[0], -q[1], -q[2], -q[3]])


def inertia_sphere(m, r):
    return [0.4 * m * r * r] * 3


def inertia_capsule(m, r, hl):
    ln = 2.0 * (hl + r)
    ixx = m * (3.0 * r * r + ln * ln) / 12.0
    return [ixx, ixx, 0.5 * m * r * r]


def inertia_box(m, he):
    k = m / 3.0
    return [k * (he[1] ** 2 + he[2] ** 2), k * (he[0] ** 2 + he[2] ** 2), k * (he[0] ** 2 + he[1] ** 2)]


class Scene:
    """One world of a custom model, with the reference's arc_phys helpers."""

    def __init__(self, model: Model, fp64: bool, dt=DT, substeps=SUB):
        self.sim = Sim(1, dt, substeps, 64, 1.0, fp64=fp64, model=model)
        self.nj = self.sim.num_joints

    def empty_terrain(self):
        self.sim.set_terrain(0, np.array([[-1e6]]), 1.0, -1e6)

    def flat(self, n, cell, height=0.0):
        self.sim.set_terrain(0, np.full((n, n), height), cell, height)

    def state(self):
        return self.sim.get_state()[0]

    def set_state(self, st):
        self.sim.set_state(st[None])

    def body(self, st, b):
        r = st[13 * b: 13 * b + 13]
        return r[0:3], r[3:7], r[7:10], r[10:13]

    def run(self, seconds, targets=None):
        n = int(seconds / self.sim.dt + 0.5)
        t = np.zeros((1, self.nj)) if targets is None else np.asarray(targets, dtype=float).reshape(1, -1)
        for _ in range(n):
            self.sim.step(t)


@pytest.fixture(params=[True, False], ids=["fp64", "fp32"])
def fp64(request):
    return request.param


def tol(fp64, t64, t32):
    return t64 if fp64 else t32


def energy(st, masses, inertias, g=(0, 0, -9.81)):
    e = 0.0
    for b, (m, I) in enumerate(zip(masses, inertias)):
        x, q, v, w = st[13 * b: 13 * b + 3], st[13 * b + 3: 13 * b + 7], st[13 * b + 7: 13 * b + 10], \
            st[13 * b + 10: 13 * b + 13]
        wl = qrot(qinv(q), w)
        e += 0.5 * m * v @ v + 0.5 * wl @ (wl * np.asarray(I)) - m * np.asarray(g) @ x
    return e


def test_free_fall(fp64):  # csrc/tests/test_phys.c:63-75
    m = Model()
    m.add_body(2.0, inertia_sphere(2.0, 0.1), [0, 0, 0])
    s = Scene(m, fp64)
    s.empty_terrain()
    st = s.state()
    st[7:10] = [1.0, 0.0, 0.0]
    s.set_state(st)
    s.run(1.0)
    x, q, v, w = s.body(s.state(), 0)
    assert abs(x[2] + 0.5 * 9.81) <= 1e-2
    assert abs(x[0] - 1.0) <= tol(fp64, 1e-9, 1e-4)
    # XPBD derives v = (x - x_prev) / h (csrc/arc_phys.c:682): in FP32 the
    # rounding of |x| ~ 5 m (2.4e-7) is amplified by 1/h = 600 every substep
    assert abs(v[2] + 9.81) <= tol(fp64, 1e-9, 2e-2)


def test_free_rotation(fp64):  # csrc/tests/test_phys.c:77-99
    m = Model()
    m.add_body(1.0, [1.0, 2.0, 3.0], [0, 0, 0])
    s = Scene(m, fp64)
    s.empty_terrain()
    s.sim.set_world_params(gravity=(0.0, 0.0, 0.0))
    st = s.state()
    st[10:13] = [0.2, 0.3, 4.0]
    s.set_state(st)
    I = np.array([1.0, 2.0, 3.0])
    x, q, v, w = s.body(st, 0)
    L0 = qrot(q, qrot(qinv(q), w) * I)
    e0 = energy(st, [1.0], [I], g=(0, 0, 0))
    s.run(5.0)
    st = s.state()
    x, q, v, w = s.body(st, 0)
    L1 = qrot(q, qrot(qinv(q), w) * I)
    e1 = energy(st, [1.0], [I], g=(0, 0, 0))
    assert np.linalg.norm(L1 - L0) / np.linalg.norm(L0) <= 0.02
    assert (e1 - e0) / e0 <= tol(fp64, 1e-6, 1e-5)
    assert (e0 - e1) / e0 <= 0.05


def test_pendulum_period(fp64):  # csrc/tests/test_phys.c:101-141
    L, mass, r, th0 = 1.0, 1.0, 0.05, 0.1
    m = Model()
    m.add_body(mass, inertia_sphere(mass, r), [0, 0, -L])
    m.add_hinge(-1, 0, [0, 0, 0], [0, 1, 0])
    s = Scene(m, fp64, dt=1.0 / 600.0, substeps=1)
    s.empty_terrain()
    s.sim.set_pose(0, [0, 0, 0], [1, 0, 0, 0], [th0])
    x, q, v, w = s.body(s.state(), 0)
    assert abs(x[0] + L * np.sin(th0)) <= tol(fp64, 1e-12, 1e-6)
    i_pivot = 0.4 * mass * r * r + mass * L * L
    period = 2.0 * np.pi * np.sqrt(i_pivot / (mass * 9.81 * L))
    e0 = energy(s.state(), [mass], [inertia_sphere(mass, r)])
    a_prev = th0
    first, last, crossings = -1.0, 0.0, 0
    tgt = np.zeros((1, 1))
    for k in range(6000):
        s.sim.step(tgt)
        a = s.sim.observe()[1][0, 0]
        if a_prev > 0.0 and a <= 0.0:
            t = (k + 1) / 600.0 - (1.0 / 600.0) * a / (a - a_prev)
            if first < 0:
                first = t
            last = t
            crossings += 1
        a_prev = a
    assert abs((last - first) / (crossings - 1) - period) <= 2e-3 * period
    e1 = energy(s.state(), [mass], [inertia_sphere(mass, r)])
    swing = mass * 9.81 * L * (1.0 - np.cos(th0))
    assert (e1 - e0) / swing <= tol(fp64, 1e-6, 1e-3)
    assert (e0 - e1) / swing <= 0.2


def test_chain_separation(fp64):  # csrc/tests/test_phys.c:143-171
    n, seg = 6, 0.3
    m = Model()
    anchors, qs, xs = [], [], []
    for i in range(n):
        mass = 1.0 - 0.9 * i / (n - 1.0)
        q = qaxis([0, 1, 0], 0.5 * np.pi)
        x = np.array([(i + 0.5) * seg, 0, 0])
        m.add_body(mass, inertia_capsule(mass, 0.03, 0.5 * seg), x, q)
        m.add_hinge(i - 1, i, [i * seg, 0, 0], [0, 1, 0])
        anchors.append(np.array([i * seg, 0.0, 0.0]))
        qs.append(q / np.linalg.norm(q))
        xs.append(x)
    r1 = [qrot(qinv(qs[i - 1]), anchors[i] - xs[i - 1]) if i > 0 else anchors[0] for i in range(n)]
    r2 = [qrot(qinv(qs[i]), anchors[i] - xs[i]) for i in range(n)]
    s = Scene(m, fp64)
    s.empty_terrain()
    maxsep = 0.0
    for _ in range(90):
        s.sim.step(np.zeros((1, n)))
        st = s.state()
        for i in range(n):
            xc, qc, _, _ = s.body(st, i)
            p2 = xc + qrot(qc, r2[i])
            if i > 0:
                xp, qp, _, _ = s.body(st, i - 1)
                p1 = xp + qrot(qp, r1[i])
            else:
                p1 = r1[0]
            maxsep = max(maxsep, np.linalg.norm(p1 - p2))
    assert maxsep <= 2e-3
    assert not s.sim.observe()[3][0]
    assert s.body(s.state(), n - 1)[0][2] <= 1e-6


def arm(fp64, gravity_on=True):
    m = Model()
    m.add_body(1.0, inertia_capsule(1.0, 0.03, 0.25), [0.25, 0, 0], qaxis([0, 1, 0], 0.5 * np.pi))
    m.add_hinge(-1, 0, [0, 0, 0], [0, 1, 0])
    s = Scene(m, fp64)
    s.empty_terrain()
    if not gravity_on:
        s.sim.set_world_params(gravity=(0.0, 0.0, 0.0))
    return s


def test_hinge_limits(fp64):  # csrc/tests/test_phys.c:173-194
    s = arm(fp64)
    lo, hi = -0.3, 0.4
    s.sim.set_joint(0, lo, hi, 0.0, 0.0, 0.0)
    amin, amax = 1e9, -1e9
    for _ in range(120):
        s.sim.step(np.zeros((1, 1)))
        a = s.sim.observe()[1][0, 0]
        amin, amax = min(amin, a), max(amax, a)
    assert amax - hi <= 5e-3
    assert lo - amin <= 5e-3
    assert abs(s.sim.observe()[1][0, 0] - hi) <= 5e-3


def test_pd_drive(fp64):  # csrc/tests/test_phys.c:196-226
    s = arm(fp64, gravity_on=False)
    s.sim.set_joint(0, 1.0, -1.0, 50.0, 2.0, 100.0)
    s.run(2.0, targets=[0.5])
    j = s.sim.observe()[1][0]
    assert abs(j[0] - 0.5) <= 1e-3
    assert abs(j[1]) <= 1e-3
    s.sim.set_world_params(gravity=(0.0, 0.0, -9.81))
    s.run(3.0, targets=[0.0])
    j = s.sim.observe()[1][0]
    assert abs(j[0] - 9.81 * 0.25 / 50.0) <= 2e-3
    assert abs(j[2] + 9.81 * 0.25) <= 0.05
    s.sim.set_joint(0, 1.0, -1.0, 50.0, 2.0, 0.2)
    s.run(6.0, targets=[0.0])
    j = s.sim.observe()[1][0]
    assert abs(abs(j[2]) - 0.2) <= 0.02
    assert j[0] > 1.2


def test_resting_sphere(fp64):  # csrc/tests/test_phys.c:228-246
    m = Model()
    m.add_body(1.0, inertia_sphere(1.0, 0.1), [0.01, 0.02, 0.5])
    m.add_sphere(0, [0, 0, 0], 0.1)
    s = Scene(m, fp64)
    s.flat(8, 0.5)
    s.run(1.0)
    maxv = 0.0
    for _ in range(60):
        s.sim.step(np.zeros((1, 0)))
        maxv = max(maxv, np.linalg.norm(s.body(s.state(), 0)[2]))
    st = s.state()
    assert abs(st[2] - 0.1) <= 1e-4
    assert maxv <= 1e-3
    assert st[13 + 7] == SUB  # touch count of the sphere


def test_sliding_friction(fp64):  # csrc/tests/test_phys.c:248-289
    he, r = np.array([0.2, 0.2, 0.05]), 0.03
    m = Model()
    m.add_body(2.0, inertia_box(2.0, he), [-4.0, 0, 0.05])
    for sx in (-1, 1):
        for sy in (-1, 1):
            m.add_sphere(0, [sx * (he[0] - r), sy * (he[1] - r), -he[2] + r], r)
    s = Scene(m, fp64)
    s.flat(32, 0.5)
    s.sim.set_world_params(mu_static=0.5, mu_dynamic=0.5)
    s.run(0.2)
    st = s.state()
    x0 = st[0]
    st[7:10] = [3.0, 0, 0]
    s.set_state(st)
    s.run(2.0)
    st = s.state()
    assert abs(st[0] - x0 - 9.0 / (2 * 0.5 * 9.81)) <= 0.05
    assert np.linalg.norm(st[7:10]) <= 5e-3
    x1, ang = st[0], np.radians(20.0)
    s.sim.set_world_params(gravity=(9.81 * np.sin(ang), 0, -9.81 * np.cos(ang)), mu_static=0.5, mu_dynamic=0.5)
    s.run(2.0)
    assert abs(s.state()[0] - x1) <= 5e-3
    s.sim.set_world_params(gravity=(9.81 * np.sin(ang), 0, -9.81 * np.cos(ang)), mu_static=0.3, mu_dynamic=0.3)
    s.run(1.0)
    assert s.state()[0] - x1 > 0.25


def test_block_terrain(fp64):  # csrc/tests/test_phys.c:291-323
    r = 0.1
    m = Model()
    for pos in ([0.5, 0.0, 0.6], [-0.12, 0.25, 0.6], [0.02, -0.75, 0.6]):
        b = m.add_body(1.0, inertia_sphere(1.0, r), pos)
        m.add_sphere(b, [0, 0, 0], r)
    s = Scene(m, fp64)
    h = np.zeros((8, 8))
    h[:, 4:] = 0.3
    s.sim.set_terrain(0, h, 0.5, 0.0)
    z = s.sim.terrain_at(np.array([0, 0]), np.array([[0.1, 0.1], [-0.1, 0.1]]))
    assert abs(z[0] - 0.3) <= 1e-7 and abs(z[1]) <= 1e-12
    s.run(3.0)
    st = s.state()
    assert abs(st[2] - 0.4) <= 1e-4 and abs(st[0] - 0.5) <= 1e-4
    assert abs(st[13 + 2] - 0.1) <= 1e-4 and st[13 + 0] <= -0.1 + 1e-4
    assert abs(st[26 + 2] - 0.4) <= 1e-3 and np.linalg.norm(st[26 + 7: 26 + 10]) <= 1e-3


def test_forward_kinematics_set_pose(fp64):  # csrc/tests/test_phys.c:325-342
    m = Model()
    bodies = [(5.0, [1, 1, 1], [0, 0, 0]), (1.0, [.1, .1, .1], [0.2, 0, -0.2]),
              (1.0, [.1, .1, .1], [0.2, 0, -0.6]), (1.0, [.1, .1, .1], [0.2, 0.1, -1.0])]
    for mass, I, pos in bodies:
        m.add_body(mass, I, pos)
    hinges = [(0, 1, [0.2, 0, 0], [1, 0, 0]), (1, 2, [0.2, 0, -0.4], [0, 1, 0]), (2, 3, [0.2, 0, -0.8], [0, 0.6, 0.8])]
    frames = []
    for p, c, anchor, axis in hinges:
        m.add_hinge(p, c, anchor, axis)
        ax = np.asarray(axis, float) / np.linalg.norm(axis)
        t = np.array([1.0, 0, 0]) if abs(ax[0]) < 0.57 else np.array([0, 1.0, 0])
        ref = np.cross(ax, t)
        ref /= np.linalg.norm(ref)
        frames.append((p, c, ax, ref, ref))  # bodies start unrotated: frames equal world vectors
    s = Scene(m, fp64)
    s.empty_terrain()
    angles = [0.3, -0.7, 1.1]
    s.sim.set_pose(0, [1, 2, 3], qaxis([0, 0, 1], 0.8), angles)
    st = s.state()
    for k, (p, c, a1, b1, b2) in enumerate(frames):
        qp, qc = st[13 * p + 3: 13 * p + 7], st[13 * c + 3: 13 * c + 7]
        a, v1, v2 = qrot(qp, a1), qrot(qp, b1), qrot(qc, b2)
        ang = np.arctan2(np.cross(v1, v2) @ a, v1 @ v2)
        assert abs(ang - angles[k]) <= tol(fp64, 1e-9, 1e-6)


@pytest.mark.parametrize("bad", [1e12, -1e300, np.nan])
def test_blow_up_is_flagged(fp64, bad):  # csrc/tests/test_phys.c:344-364
    m = Model()
    m.add_body(1.0, inertia_sphere(1.0, 0.1), [0.0, 0.0, 0.05])
    m.add_sphere(0, [0, 0, 0], 0.1)
    s = Scene(m, fp64)
    s.flat(8, 0.5)
    st = s.state()
    st[0] = bad
    s.set_state(st)
    s.sim.step(np.zeros((1, 0)))
    assert s.sim.observe()[3][0] == 1
    z = s.sim.terrain_at(np.array([0]), np.array([[bad, bad]]))
    assert z[0] == 0.0


def test_ball_falls_into_the_void(fp64):  # csrc/tests/test_robot.c:128-148
    m = Model()
    m.add_body(1.0, inertia_sphere(1.0, 0.1), [0.0, 0.0, 1.0])
    m.add_sphere(0, [0, 0, 0], 0.1)
    s = Scene(m, fp64)
    from oracle.oracle import oracle_terrain
    h, geom = oracle_terrain(32, 0.4, 0.5, 9)
    s.sim.set_terrain(0, h, 0.4, -100.0)
    edge = geom[2] + 32 * 0.4
    st = s.state()
    st[0] = edge - 1.0
    st[7:10] = [4.0, 0.0, 0.0]
    s.set_state(st)
    s.run(3.0)
    st = s.state()
    assert st[0] > edge
    assert st[2] <= -2.0
