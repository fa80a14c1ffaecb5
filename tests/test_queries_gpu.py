"""World queries on the GPU against the reference, bit for bit, on seeded
stepped worlds (reference src/world.cpp:1081-1416):

- m3d_world_ray_cast / _filtered: the grid walk over both tiers and the
  oversized lists, first hit by fraction;
- m3d_world_sphere_cast: start overlaps, inflated ray casts of spheres and
  capsules, conservative advancement against boxes, nearest hit with the
  reference's index order on ties; and m3d_gpu_sphere_cast_noalloc;
- m3d_world_overlap_aabb: the callback sequence (body ids in index order)
  and the early stop when the callback returns false.

Queries run both right after a step and after a destroy/spawn churn without
a step, when the broadphase is stale and the query refreshes it first (which
also changes what the next step does - the worlds must stay in lockstep).
"""
import ctypes as C

import numpy as np
import pytest

from melon3d_b200 import api, harness

from . import _util as U

pytestmark = pytest.mark.gpu


def _bits(r):
    return (bool(r.hit), r.body.index, r.body.generation, np.float32(r.fraction).tobytes(),
            np.array([r.point.x, r.point.y, r.point.z], np.float32).tobytes(),
            np.array([r.normal.x, r.normal.y, r.normal.z], np.float32).tobytes())


def _rays(rng, count):
    out = []
    for k in range(count):
        x, z = rng.uniform(-48.0, 48.0, 2)
        if k % 3 == 0:
            o, t = (x, rng.uniform(0.0, 8.0), z), tuple(rng.normal(size=3) * 30.0)
        else:
            o, t = (x, 65.0, z), (rng.uniform(-10, 10), -70.0, rng.uniform(-10, 10))
        mask = 0xFFFFFFFF if k % 4 else (0x1 if k % 8 else 0x0)
        out.append((api.Vec3(*map(float, o)), api.Vec3(*map(float, t)), mask))
    return out


def _sphere_casts(rng, count):
    out = []
    for k in range(count):
        x, z = rng.uniform(-48.0, 48.0, 2)
        r = float(rng.uniform(0.05, 2.0))
        if k % 5 == 0:  # short casts near the ground: start overlaps and box advancement
            o, t = (x, rng.uniform(0.0, 2.0), z), tuple(rng.normal(size=3) * 2.0)
        elif k % 7 == 0:  # zero-length cast
            o, t = (x, rng.uniform(0.0, 3.0), z), (0.0, 0.0, 0.0)
        else:
            o, t = (x, 65.0, z), (rng.uniform(-10, 10), -70.0, rng.uniform(-10, 10))
        mask = 0xFFFFFFFF if k % 6 else 0x1
        out.append((api.Vec3(*map(float, o)), r, api.Vec3(*map(float, t)), mask))
    return out


def _overlap(lib, world, box, stop_after=None):
    seen = []

    @api.OverlapFn
    def cb(bid, ctx):
        seen.append((bid.index, bid.generation))
        return stop_after is None or len(seen) < stop_after

    lib.m3d_world_overlap_aabb(world, box, cb, None)
    return seen


def _boxes(rng, count):
    out = []
    for _ in range(count):
        c = np.array([rng.uniform(-45, 45), rng.uniform(-1, 8), rng.uniform(-45, 45)])
        h = rng.uniform(0.2, 6.0, 3)
        out.append(api.AABB(api.Vec3(*map(float, c - h)), api.Vec3(*map(float, c + h))))
    return out


def _compare_queries(ref, g, wr, wg, rng, tag):
    for o, t, mask in _rays(rng, 150):
        a = ref.m3d_world_ray_cast_filtered(wr, o, t, mask)
        b = g.m3d_world_ray_cast_filtered(wg, o, t, mask)
        assert _bits(a) == _bits(b), "%s: ray %s" % (tag, (o.tup(), t.tup(), mask))
        if mask == 0xFFFFFFFF:
            assert _bits(ref.m3d_world_ray_cast(wr, o, t)) == _bits(b)
    hits = 0
    for o, r, t, mask in _sphere_casts(rng, 150):
        a = ref.m3d_world_sphere_cast(wr, o, r, t, mask)
        b = g.m3d_world_sphere_cast(wg, o, r, t, mask)
        assert _bits(a) == _bits(b), "%s: sphere cast %s" % (tag, (o.tup(), r, t.tup(), mask))
        if hasattr(g, "m3d_gpu_sphere_cast_noalloc"):
            out = api.RayResult()
            rc = g.m3d_gpu_sphere_cast_noalloc(wg, o, r, t, mask, C.byref(out))
            assert rc == api.GPU_OK and _bits(out) == _bits(a)
        hits += a.hit
    assert hits > 20
    found = 0
    for k, box in enumerate(_boxes(rng, 60)):
        stop = None if k % 3 else 2
        a = _overlap(ref, wr, box, stop)
        b = _overlap(g, wg, box, stop)
        assert a == b, "%s: overlap %d" % (tag, k)
        found += len(a)
    assert found > 20


@pytest.mark.parametrize("seed", [5, 12])
def test_queries_match_the_reference(seed):
    ref, g = U.oracle_cr(), U.gpu()
    sr = harness.Scene(ref, harness.RAIN, seed, 4000, 40)
    sg = harness.Scene(g, harness.RAIN, seed, 4000, 40)
    rng = np.random.default_rng(seed)
    try:
        for step in range(90):
            sr.run(1)
            sg.run(1)
            if step in (0, 45, 89):
                _compare_queries(ref, g, sr.world, sg.world, rng, "after step %d" % step)
        # churn without a step: the queries refresh the stale broadphase
        sr.churn()
        sg.churn()
        # the destroys' end events (touching contacts of each destroyed body)
        er, eg = U.events(ref, sr.world), U.events(g, sg.world)
        assert len(er[1]) > 0
        d = U.diff_events(er, eg)
        assert d is None, d
        _compare_queries(ref, g, sr.world, sg.world, rng, "after churn")
        for step in range(5):
            sr.step_only()
            sg.step_only()
        d = U.diff_bodies(U.bodies(ref, sr.world), U.bodies(g, sg.world))
        assert d is None, d
        d = U.diff_contacts(U.contacts(ref, sr.world), U.contacts(g, sg.world))
        assert d is None, d
    finally:
        sr.close()
        sg.close()


def test_queries_on_a_sleeping_world():
    # the sleeping-world fast path leaves the broadphase as the reference's
    ref, g = U.oracle(), U.gpu()
    sr = harness.Scene(ref, harness.SETTLED_STACKS, 1, 20, 20, 2)
    sg = harness.Scene(g, harness.SETTLED_STACKS, 1, 20, 20, 2)
    rng = np.random.default_rng(3)
    try:
        sr.run(70)
        sg.run(70)
        assert g.m3d_gpu_fast_path_steps(sg.world) > 0
        for o, t, mask in _rays(rng, 100):
            o = api.Vec3(o.x * 0.3, o.y, o.z * 0.3)
            assert _bits(ref.m3d_world_ray_cast_filtered(sr.world, o, t, mask)) == \
                _bits(g.m3d_world_ray_cast_filtered(sg.world, o, t, mask))
        for box in _boxes(rng, 40):
            assert _overlap(ref, sr.world, box) == _overlap(g, sg.world, box)
    finally:
        sr.close()
        sg.close()
