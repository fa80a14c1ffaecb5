"""Adjoint of recorded steps (m3d_gpu_step_backward, include/melon3d_gpu.h).

- the tape replay (the forward half of the adjoint) reproduces the world's
  own states bit for bit, single worlds and batches, sleep on and off;
- the regenerating replay (the tape's discrete record only, every manifold
  regenerated at its recorded generation events) reproduces the world bit for
  bit in float: the tape holds every dependence of the steps on the states;
- the adjoint equals central differences (h = 1e-6, double) of the
  regenerating replay for initial linear and angular velocities, masses,
  friction and restitution: the exact derivative of the branch the forward
  took;
- on smooth motions (rolling, sliding) the adjoint agrees with central
  differences (h = 1e-3) of the engine itself;
- the GPU adjoint agrees with the FP64 host evaluation of the same adjoint;
- an unsupported tape (joints) is refused with M3D_GPU_ERR_UNSUPPORTED.

Losses: weighted sums of final positions, or the differentiable-batch loss
(sum over worlds of |centroid - target|^2) through a thin
torch.autograd.Function whose backward calls the C ABI.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from melon3d_b200 import api, harness
from tests._util import bodies, gpu

pytestmark = pytest.mark.gpu

FP = C.POINTER(C.c_float)
DP = C.POINTER(C.c_double)


def _p(a, t=FP):
    return None if a is None else a.ctypes.data_as(t)


def state(lib, world):
    b = bodies(lib, world)
    return (b["position"].copy(), b["rotation"].copy(), b["linearVelocity"].copy(),
            b["angularVelocity"].copy(), b["inUse"] != 0)


def replay(lib, world):
    n = lib.m3d_gpu_body_capacity(world)
    pos, rot = np.zeros((n, 3), np.float32), np.zeros((n, 4), np.float32)
    vel, ang = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32)
    rc = lib.m3d_gpu_tape_replay(world, _p(pos), _p(rot), _p(vel), _p(ang), n)
    assert rc == api.GPU_OK, rc
    return pos, rot, vel, ang


def backward(lib, world, dpos, fp64=False):
    """Gradients of the recorded trajectory for a position adjoint `dpos`."""
    n = lib.m3d_gpu_body_capacity(world)
    dt = np.float64 if fp64 else np.float32
    t = DP if fp64 else FP
    g = {"pos": np.zeros((n, 3), dt), "rot": np.zeros((n, 4), dt), "vel": np.zeros((n, 3), dt),
         "ang": np.zeros((n, 3), dt), "mass": np.zeros(n, dt), "mu": np.zeros(n, dt), "e": np.zeros(n, dt)}
    d = np.ascontiguousarray(dpos, dtype=dt)
    fn = lib.m3d_gpu_step_backward_fp64_host if fp64 else lib.m3d_gpu_step_backward
    rc = fn(world, _p(d, t), None, None, None, _p(g["pos"], t), _p(g["rot"], t), _p(g["vel"], t), _p(g["ang"], t),
            _p(g["mass"], t), _p(g["mu"], t), _p(g["e"], t), n)
    return rc, g


def regenerate(lib, world, dbl, dvel=None, dang=None, dmass=None, dmu=None, de=None):
    """Final states of the regenerating replay (float or double)."""
    n = lib.m3d_gpu_body_capacity(world)
    out = [np.zeros((n, 3)), np.zeros((n, 4)), np.zeros((n, 3)), np.zeros((n, 3))]
    args = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (dvel, dang, dmass, dmu, de)]
    rc = lib.m3d_gpu_tape_regenerate_host(world, 1 if dbl else 0, *[_p(a, DP) for a in args],
                                          *[_p(o, DP) for o in out], n)
    assert rc == api.GPU_OK, rc
    return out


def centroid_loss(pos, slots, targets):
    loss = 0.0
    dpos = np.zeros_like(pos, dtype=np.float64)
    for k, s in enumerate(slots):
        c = pos[s].astype(np.float64).mean(axis=0)
        r = c - targets[k]
        loss += float(r @ r)
        dpos[s] += 2.0 * r / len(s)
    return loss, dpos


class FinalPositions(torch.autograd.Function):
    """Final positions of a recorded trajectory as a function of the initial
    velocities, masses, friction and restitution; backward calls
    m3d_gpu_step_backward."""

    @staticmethod
    def forward(ctx, v0, mass, mu, e, lib, world, final_pos):
        ctx.lib, ctx.world = lib, world
        return torch.from_numpy(final_pos.astype(np.float32))

    @staticmethod
    def backward(ctx, dpos):
        rc, g = backward(ctx.lib, ctx.world, dpos.detach().cpu().numpy())
        assert rc == api.GPU_OK, rc
        return (torch.from_numpy(g["vel"]), torch.from_numpy(g["mass"]), torch.from_numpy(g["mu"]),
                torch.from_numpy(g["e"]), None, None, None)


def _incline(lib, seed, count=0, sleep=False):
    return harness.Scene(lib, harness.INCLINE, seed=seed, a=count, b=1 if sleep else 0)


def _relerr(a, b):
    a, b = np.asarray(a, np.float64).ravel(), np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def _same_bits(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


@pytest.mark.parametrize("seed,sleep,steps", [(1, False, 40), (2, False, 40), (3, True, 150)])
def test_replay_reproduces_the_world(seed, sleep, steps):
    lib = gpu()
    sc = _incline(lib, seed, sleep=sleep)
    assert lib.m3d_gpu_tape_begin(sc.world, 10) == api.GPU_OK
    for _ in range(steps):
        sc.step_only(4)
    why = C.create_string_buffer(200)
    assert lib.m3d_gpu_tape_supported(sc.world, why, 200) == 1, why.value
    assert lib.m3d_gpu_tape_steps(sc.world) == steps
    pos, rot, vel, ang, live = state(lib, sc.world)
    rp, rr, rv, ra = replay(lib, sc.world)
    for name, a, b in (("position", pos, rp), ("rotation", rot, rr), ("velocity", vel, rv), ("angular", ang, ra)):
        assert _same_bits(a[live], b[live]), name
    if sleep:
        assert lib.m3d_world_profile(sc.world).awakeBodyCount < 64  # some bodies fell asleep
    sc.close()


def test_replay_reproduces_a_batch():
    lib = gpu()
    scenes = [_incline(lib, 100 + k) for k in range(8)]
    arr = (C.c_void_p * len(scenes))(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, len(scenes))
    assert batch
    assert lib.m3d_gpu_tape_begin(batch, 10) == api.GPU_OK
    for _ in range(30):
        lib.m3d_world_step(batch, 1.0 / 60.0, 4)
    pos, rot, vel, ang, live = state(lib, batch)
    rp, rr, rv, ra = replay(lib, batch)
    for a, b in ((pos, rp), (rot, rr), (vel, rv), (ang, ra)):
        assert _same_bits(a[live], b[live])
    lib.m3d_world_destroy(batch)
    for s in scenes:
        s.close()


def test_batch_adjoint_through_autograd():
    """The differentiable-batch loss at reduced world count: one world's
    gradient taken from the batch equals that world's gradient taken alone,
    bit for bit."""
    lib = gpu()
    seeds = [200 + k for k in range(6)]
    scenes = [_incline(lib, s) for s in seeds]
    ids = [s.dynamic_ids() for s in scenes]
    arr = (C.c_void_p * len(scenes))(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, len(scenes))
    assert lib.m3d_gpu_tape_begin(batch, 10) == api.GPU_OK
    for _ in range(40):
        lib.m3d_world_step(batch, 1.0 / 60.0, 4)
    n = lib.m3d_gpu_body_capacity(batch)
    slots = [np.array([lib.m3d_gpu_batch_first_body(batch, k) + i.index for i in ids[k]]) for k in range(len(seeds))]
    targets = np.random.default_rng(7).normal(size=(len(seeds), 3))
    pos = state(lib, batch)[0]
    v0 = torch.zeros((n, 3), requires_grad=True)
    mass = torch.zeros(n, requires_grad=True)
    mu = torch.zeros(n, requires_grad=True)
    e = torch.zeros(n, requires_grad=True)
    final = FinalPositions.apply(v0, mass, mu, e, lib, batch, pos)
    loss = 0
    for k, s in enumerate(slots):
        c = final[torch.from_numpy(s)].double().mean(dim=0)
        loss = loss + ((c - torch.from_numpy(targets[k])) ** 2).sum()
    loss.backward()
    gb = v0.grad.numpy()
    k = 2
    alone = _incline(lib, seeds[k])
    lib.m3d_gpu_tape_begin(alone.world, 10)
    for _ in range(40):
        alone.step_only(4)
    pa = state(lib, alone.world)[0]
    sa = np.array([i.index for i in ids[k]])
    assert _same_bits(pa[sa], pos[slots[k]])
    _, dpa = centroid_loss(pa, [sa], targets[k:k + 1])
    rc, ga = backward(lib, alone.world, dpa)
    assert rc == api.GPU_OK
    # bit for bit: the batch runs each world's islands exactly as alone
    assert _same_bits(gb[slots[k]], ga["vel"][sa])
    alone.close()
    lib.m3d_world_destroy(batch)
    for s in scenes:
        s.close()


# ---- small scenes built through the API -------------------------------------------

_TH = np.deg2rad(25.0)


def _build_fd_world(lib, spec, theta, dv=None, dw=None):
    """A small incline world from an explicit per-body spec; dv / dw perturb
    one initial velocity component: (body, component, delta)."""
    wd = lib.m3d_world_def_default()
    wd.enableSleep = False
    w = lib.m3d_world_create(C.byref(wd))
    q = api.Quat(0.0, 0.0, float(np.sin(0.5 * theta)), float(np.cos(0.5 * theta)))
    gd = lib.m3d_body_def_default()
    gd.type = api.BODY_STATIC
    gd.orientation = q
    gs = lib.m3d_shape_def_default()
    gs.type = api.SHAPE_BOX
    gs.halfExtents = api.Vec3(8.0, 0.25, 5.0)
    gs.friction = 1.0
    gs.restitution = 0.0
    lib.m3d_body_create(w, C.byref(gd), C.byref(gs))
    ids = []
    c, s = np.cos(theta), np.sin(theta)
    for i, b in enumerate(spec):
        bd = lib.m3d_body_def_default()
        bd.type = api.BODY_DYNAMIC
        lx, ly, lz = b["local"]
        bd.position = api.Vec3(float(c * lx - s * ly), float(s * lx + c * ly), float(lz))
        bd.orientation = q
        v = np.array(b["v"], np.float64)
        wv = np.array(b.get("w", [0.0, 0.0, 0.0]), np.float64)
        if dv is not None and dv[0] == i:
            v[dv[1]] += dv[2]
        if dw is not None and dw[0] == i:
            wv[dw[1]] += dw[2]
        bd.linearVelocity = api.Vec3(*[float(x) for x in v])
        bd.angularVelocity = api.Vec3(*[float(x) for x in wv])
        sd = lib.m3d_shape_def_default()
        sd.type = b["type"]
        if b["type"] == api.SHAPE_BOX:
            sd.halfExtents = api.Vec3(b["size"], b["size"], b["size"])
        else:
            sd.radius = b["size"]
        sd.friction = float(b["mu"])
        sd.restitution = float(b["e"])
        ids.append(lib.m3d_body_create(w, C.byref(bd), C.byref(sd)))
    return w, ids


def _slope(vx, vz=0.0):
    """A velocity along the incline's slope (its local x), world frame."""
    return [vx * np.cos(_TH), vx * np.sin(_TH), vz]


def _on(x, size, z=0.0, lift=-0.001):
    return (x, 0.25 + size + lift, z)


B, S = api.SHAPE_BOX, api.SHAPE_SPHERE
# Smooth motions: rolling, sliding, pair collisions, a box landing on a box.
SCENES = {
    "sphere rolling": ([{"type": S, "size": 0.2, "local": _on(0, 0.2), "v": [0.3, 0.0, 0.2], "w": [1.0, -2.0, 3.0],
                         "mu": 0.8, "e": 0.1}], 8),
    "box sliding": ([{"type": B, "size": 0.2, "local": _on(0, 0.2), "v": [0.3, 0.0, 0.2], "w": [0.5, 1.0, -0.7],
                      "mu": 0.2, "e": 0.1}], 8),
    "spheres colliding": ([
        {"type": S, "size": 0.2, "local": _on(-0.42, 0.2), "v": _slope(1.0, 0.05), "mu": 0.6, "e": 0.2},
        {"type": S, "size": 0.2, "local": _on(0.0, 0.2, 0.03), "v": _slope(0.0), "mu": 0.5, "e": 0.15}], 8),
    "boxes colliding": ([
        {"type": B, "size": 0.2, "local": _on(-0.42, 0.2), "v": _slope(1.2, 0.05), "mu": 0.25, "e": 0.2},
        {"type": B, "size": 0.2, "local": _on(0.0, 0.2, 0.03), "v": _slope(0.0), "mu": 0.3, "e": 0.15}], 20),
    "box landing on box": ([
        {"type": B, "size": 0.2, "local": _on(0.0, 0.2), "v": _slope(0.0), "mu": 0.9, "e": 0.05},
        {"type": B, "size": 0.15, "local": (0.03, 0.25 + 0.4 + 0.15 + 0.01, 0.02), "v": [0.1, -0.3, 0.05], "mu": 0.8,
         "e": 0.0}], 20),
}


def _recorded(lib, name):
    spec, steps = SCENES[name]
    w, ids = _build_fd_world(lib, spec, _TH)
    assert lib.m3d_gpu_tape_begin(w, 10) == api.GPU_OK
    for _ in range(steps):
        lib.m3d_world_step(w, 1.0 / 60.0, 4)
    why = C.create_string_buffer(200)
    assert lib.m3d_gpu_tape_supported(w, why, 200) == 1, why.value
    return w, np.array([i.index for i in ids]), spec, steps


@pytest.mark.parametrize("name", list(SCENES))
def test_regenerating_replay_reproduces_the_world(name):
    lib = gpu()
    w, s, _, _ = _recorded(lib, name)
    pos, rot, vel, ang, live = state(lib, w)
    r = regenerate(lib, w, False)
    for a, b in ((pos, r[0]), (rot, r[1]), (vel, r[2]), (ang, r[3])):
        assert _same_bits(a[live], b[live])
    lib.m3d_world_destroy(w)


@pytest.mark.parametrize("seed,sleep,steps", [(1, False, 40), (3, True, 150)])
def test_regenerating_replay_reproduces_the_incline_world(seed, sleep, steps):
    lib = gpu()
    sc = _incline(lib, seed, sleep=sleep)
    assert lib.m3d_gpu_tape_begin(sc.world, 10) == api.GPU_OK
    for _ in range(steps):
        sc.step_only(4)
    pos, rot, vel, ang, live = state(lib, sc.world)
    r = regenerate(lib, sc.world, False)
    for a, b in ((pos, r[0]), (rot, r[1]), (vel, r[2]), (ang, r[3])):
        assert _same_bits(a[live], b[live])
    sc.close()


def _directional(lib, w, s, u, kind, d, h):
    """Central difference (double regenerating replay) of sum(u * final
    positions of s) along the perturbation direction d."""
    n = lib.m3d_gpu_body_capacity(w)
    full = np.zeros((n, 3) if kind in ("vel", "ang") else n)
    full[s] = d
    kw = {"vel": "dvel", "ang": "dang", "mass": "dmass", "mu": "dmu", "e": "de"}[kind]
    pp = regenerate(lib, w, True, **{kw: h * full})[0]
    pm = regenerate(lib, w, True, **{kw: -h * full})[0]
    return float(((pp - pm)[s] * u).sum() / (2 * h))


@pytest.mark.parametrize("name", list(SCENES))
def test_adjoint_is_the_derivative_of_the_recorded_branch(name):
    """GPU and FP64 adjoints against central differences (double) of the
    regenerating replay: initial velocities, masses, friction and restitution
    along random directions.  The tolerance is relative to the gradient's
    scale (the largest directional derivative): rounding-level branch ties (a
    constraint met exactly, re-checked in the next iteration) stay inside
    2e-3 of it, float accumulation in the GPU adjoint inside 3e-3."""
    lib = gpu()
    w, s, spec, _ = _recorded(lib, name)
    n = lib.m3d_gpu_body_capacity(w)
    rng = np.random.default_rng(7)
    u = rng.normal(size=(len(s), 3))
    dpos = np.zeros((n, 3))
    dpos[s] = u
    rc, g = backward(lib, w, dpos)
    assert rc == api.GPU_OK
    rc, g64 = backward(lib, w, dpos, fp64=True)
    assert rc == api.GPU_OK
    checks = []
    for kind in ("vel", "vel", "vel", "ang", "ang", "mass", "mu", "e"):
        d = rng.normal(size=(len(s), 3) if kind in ("vel", "ang") else len(s))
        h = 1e-6 if kind != "mass" else 1e-4  # masses are tens of kg
        fd = _directional(lib, w, s, u, kind, d, h)
        checks.append((kind, fd, float((g[kind][s] * d).sum()), float((g64[kind][s] * d).sum())))
    scale = max(abs(c[1]) for c in checks)
    assert scale > 0
    for kind, fd, ad, ad64 in checks:
        assert abs(ad64 - fd) <= 2e-3 * scale, (name, kind, fd, ad64, scale)
        assert abs(ad - fd) <= 3e-3 * scale, (name, kind, fd, ad, scale)
    lib.m3d_world_destroy(w)


def _engine_loss(lib, spec, steps, u, **pert):
    w, ids = _build_fd_world(lib, spec, _TH, **pert)
    for _ in range(steps):
        lib.m3d_world_step(w, 1.0 / 60.0, 4)
    pos = state(lib, w)[0]
    s = np.array([i.index for i in ids])
    lib.m3d_world_destroy(w)
    return float((pos[s].astype(np.float64) * u).sum())


@pytest.mark.parametrize("name", ["sphere rolling", "box sliding"])
def test_adjoint_matches_engine_central_differences(name):
    """Against the engine's own forward (float), central differences with
    h = 1e-3 per initial linear velocity component: on these motions no
    contact branch flips within +-h, so the engine's loss is smooth there (on
    a collision, the restitution and speculative-contact tests do flip within
    +-1e-3, and the engine's loss is not differentiable at that scale).
    Measured: 0.7 % (rolling) and 1.0 % (sliding) of the largest derivative,
    above the float rounding of the engine's loss (about 5e-5 after division by
    2h): the engine's differences at h = 1e-3 are not yet the derivative, so
    the tolerance is 1e-2 of it plus 2e-4."""
    lib = gpu()
    w, s, spec, steps = _recorded(lib, name)
    n = lib.m3d_gpu_body_capacity(w)
    u = np.random.default_rng(3).normal(size=(len(s), 3))
    dpos = np.zeros((n, 3))
    dpos[s] = u
    rc, g = backward(lib, w, dpos)
    assert rc == api.GPU_OK
    lib.m3d_world_destroy(w)
    h = 1e-3
    for key, arg in (("vel", "dv"),):
        fd = np.zeros((len(s), 3))
        for i in range(len(s)):
            for k in range(3):
                fd[i, k] = (_engine_loss(lib, spec, steps, u, **{arg: (i, k, h)}) -
                            _engine_loss(lib, spec, steps, u, **{arg: (i, k, -h)})) / (2 * h)
        adj = g[key][s]
        err = np.abs(adj - fd).max()
        print(name, key, "max |adjoint - central difference| = %.3g, max |derivative| = %.3g" % (err, np.abs(fd).max()))
        assert err <= 1e-2 * np.abs(fd).max() + 2e-4, (name, key, adj.tolist(), fd.tolist())


@pytest.mark.parametrize("name", list(SCENES))
def test_gpu_adjoint_matches_fp64_host(name):
    lib = gpu()
    w, s, _, _ = _recorded(lib, name)
    n = lib.m3d_gpu_body_capacity(w)
    dpos = np.zeros((n, 3))
    dpos[s] = np.random.default_rng(5).normal(size=(len(s), 3))
    rc, g = backward(lib, w, dpos)
    rc64, g64 = backward(lib, w, dpos, fp64=True)
    assert rc == rc64 == api.GPU_OK
    # The gradients of the parameters (initial velocities, masses, friction,
    # restitution).  Initial-pose gradients also pass through the generation
    # of the first step's manifolds, where the float and the double
    # evaluation can take different branches on near ties (aligned boxes: SAT
    # edge axes at the parallel cutoff); the float one is the engine's.
    a = np.concatenate([g[k][s].ravel() for k in ("vel", "ang", "mass", "mu", "e")])
    b = np.concatenate([g64[k][s].ravel() for k in ("vel", "ang", "mass", "mu", "e")])
    assert _relerr(a, b) <= 1e-3
    lib.m3d_world_destroy(w)


def test_joints_make_the_tape_unsupported():
    lib = gpu()
    sc = _incline(lib, 31, count=8)
    ids = sc.dynamic_ids()
    jd = api.BallJointDef()
    jd.bodyA, jd.bodyB = ids[0], ids[1]
    jd.localAnchorA = api.Vec3(0.4, 0.0, 0.0)
    jd.localAnchorB = api.Vec3(-0.4, 0.0, 0.0)
    lib.m3d_joint_create_ball(sc.world, C.byref(jd))
    assert lib.m3d_gpu_tape_begin(sc.world, 10) == api.GPU_OK
    for _ in range(5):
        sc.step_only(4)
    why = C.create_string_buffer(200)
    assert lib.m3d_gpu_tape_supported(sc.world, why, 200) == 0
    assert b"joint" in why.value, why.value
    n = lib.m3d_gpu_body_capacity(sc.world)
    rc, _ = backward(lib, sc.world, np.zeros((n, 3), np.float32))
    assert rc == api.GPU_ERR_UNSUPPORTED
    lib.m3d_gpu_tape_end(sc.world)
    assert lib.m3d_gpu_tape_steps(sc.world) == 0
    sc.close()


def _recorded_incline_batch(lib, seeds, steps):
    scenes = [_incline(lib, s) for s in seeds]
    arr = (C.c_void_p * len(scenes))(*[s.world for s in scenes])
    batch = lib.m3d_gpu_batch_create(arr, len(scenes))
    for s in scenes:
        s.close()
    assert lib.m3d_gpu_tape_begin(batch, 10) == api.GPU_OK
    for _ in range(steps):
        lib.m3d_world_step(batch, 1.0 / 60.0, 4)
    return batch


def test_warp_islands_give_the_one_thread_result():
    """Islands of 8+ contacts are replayed and reversed by a whole warp (lanes
    over one dependency level of contacts at a time).  The same recording
    with every island on one thread (M3D_TAPE_WARP_CONTACTS=0, read when the
    tape opens) must give the same replay states and gradients bit for bit."""
    import os
    lib = gpu()
    seeds = [300 + k for k in range(12)]
    results = []
    old = os.environ.get("M3D_TAPE_WARP_CONTACTS")
    try:
        for setting in (None, "0"):
            if setting is None:
                os.environ.pop("M3D_TAPE_WARP_CONTACTS", None)
            else:
                os.environ["M3D_TAPE_WARP_CONTACTS"] = setting
            batch = _recorded_incline_batch(lib, seeds, 50)
            warp = lib.m3d_gpu_tape_warp_islands(batch)
            rep = replay(lib, batch)
            n = lib.m3d_gpu_body_capacity(batch)
            dpos = np.random.default_rng(3).normal(size=(n, 3)).astype(np.float32)
            rc, g = backward(lib, batch, dpos)
            assert rc == api.GPU_OK, rc
            results.append((warp, rep, g))
            lib.m3d_world_destroy(batch)
    finally:
        if old is None:
            os.environ.pop("M3D_TAPE_WARP_CONTACTS", None)
        else:
            os.environ["M3D_TAPE_WARP_CONTACTS"] = old
    (w_warp, rep_w, g_w), (w_one, rep_1, g_1) = results
    assert w_warp > 0, "no island reached the warp threshold: the warp path was not exercised"
    assert w_one == 0
    for a, b in zip(rep_w, rep_1):
        assert _same_bits(a, b)
    for k in ("pos", "rot", "vel", "ang", "mass", "mu", "e"):
        assert _same_bits(g_w[k], g_1[k]), k


def _world_loss(pos, s, target):
    c = pos[s].astype(np.float64).mean(axis=0)
    r = c - target
    return float(r @ r), 2.0 * r / len(s)


def _incline_engine_loss(lib, seed, steps, s, target, dv):
    sc = _incline(lib, seed)
    for k, i in enumerate(sc.dynamic_ids()):
        v = lib.m3d_body_linear_velocity(sc.world, i)
        lib.m3d_body_set_linear_velocity(sc.world, i, api.Vec3(v.x + dv[k, 0], v.y + dv[k, 1], v.z + dv[k, 2]))
    for _ in range(steps):
        sc.step_only(4)
    pos = state(lib, sc.world)[0]
    sc.close()
    return _world_loss(pos, s, target)[0]


def test_adjoint_agreement_by_horizon_on_config5_worlds():
    """Config-5 incline worlds (64 bodies), loss |centroid - target|^2,
    horizons 10/20/40/120 steps: the adjoint's directional derivative along a
    random initial-velocity direction against (a) central differences of the
    double-precision regenerating replay (h = 1e-6, the exact derivative of
    the recorded branch) and (b) central differences of the engine (h = 1e-3,
    and 2e-3 for the engine against itself).  Printed as a table; asserted:
    at 10 steps some world agrees with the exact branch derivative to 1e-3,
    and the gradient grows with the horizon (the engine's loss is not smooth
    at the 1e-3 scale on these worlds, see the table)."""
    lib = gpu()
    rel = lambda a, b: abs(a - b) / max(abs(a), abs(b), 1e-30)  # noqa: E731
    rows = []
    for steps in (10, 20, 40, 120):
        for seed in (1, 2, 3):
            sc = _incline(lib, seed)
            s = np.array([i.index for i in sc.dynamic_ids()])
            assert lib.m3d_gpu_tape_begin(sc.world, 10) == api.GPU_OK
            for _ in range(steps):
                sc.step_only(4)
            target = np.random.default_rng(100 + seed).normal(size=3)
            _, dc = _world_loss(state(lib, sc.world)[0], s, target)
            n = lib.m3d_gpu_body_capacity(sc.world)
            dpos = np.zeros((n, 3))
            dpos[s] = dc
            rc, g = backward(lib, sc.world, dpos)
            assert rc == api.GPU_OK
            u = np.random.default_rng(seed * 7 + steps).normal(size=(len(s), 3))
            ad = float((g["vel"][s] * u).sum())
            full = np.zeros((n, 3))
            full[s] = u
            h6 = 1e-6
            lp = _world_loss(regenerate(lib, sc.world, True, dvel=h6 * full)[0], s, target)[0]
            lm = _world_loss(regenerate(lib, sc.world, True, dvel=-h6 * full)[0], s, target)[0]
            exact = (lp - lm) / (2 * h6)
            sc.close()
            eng = {h: (_incline_engine_loss(lib, seed, steps, s, target, h * u) -
                       _incline_engine_loss(lib, seed, steps, s, target, -h * u)) / (2 * h) for h in (1e-3, 2e-3)}
            rows.append((steps, seed, abs(ad), rel(ad, exact), rel(ad, eng[1e-3]), rel(eng[1e-3], eng[2e-3])))
    print("horizon seed |g.u| adjoint-vs-exact-branch adjoint-vs-engine(h=1e-3) engine(1e-3)-vs-engine(2e-3)")
    for r in rows:
        print("%4d %3d %10.4g %10.3g %10.3g %10.3g" % r)
    assert min(r[3] for r in rows if r[0] == 10) <= 1e-3
    mags = {steps: np.median([r[2] for r in rows if r[0] == steps]) for steps in (10, 120)}
    assert mags[120] > 100.0 * mags[10]
