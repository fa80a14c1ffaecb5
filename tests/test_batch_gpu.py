"""A batch of worlds (m3d_gpu_batch_create) against the same worlds stepped
one at a time: every world's bodies and contacts, step by step, bit for bit.
Worlds come from the batched-worlds scene generator (own ground box, 16-512
bodies of the rain distributions, 0-4 ball/hinge joints).  Also checked
against the reference itself for a few worlds."""
import ctypes as C

import numpy as np
import pytest

from melon3d_b200 import harness

from . import _util as U

pytestmark = pytest.mark.gpu


def _worlds(lib, seeds, a=0, b=0):
    return [harness.Scene(lib, harness.BATCH_WORLD, s, a, b) for s in seeds]


def _batch(g, scenes):
    arr = (C.c_void_p * len(scenes))(*[s.world for s in scenes])
    b = g.m3d_gpu_batch_create(arr, len(scenes))
    assert b, "batch creation failed"
    return b


def _world_contacts(cb, f0, f1):
    sel = (cb["bodyA"] >= f0) & (cb["bodyA"] < f1)
    out = cb[sel].copy()
    out["bodyA"] -= f0
    out["bodyB"] -= f0
    return out


def _compare(g, ref_lib, batch, scenes, step):
    bb = U.bodies(g, batch)
    cb = U.contacts(g, batch)
    for k, s in enumerate(scenes):
        f0, f1 = g.m3d_gpu_batch_first_body(batch, k), g.m3d_gpu_batch_first_body(batch, k + 1)
        d = U.diff_bodies(U.bodies(ref_lib, s.world), bb[f0:f1])
        assert d is None, "step %d world %d: %s" % (step, k, d)
        d = U.diff_contacts(U.contacts(ref_lib, s.world), _world_contacts(cb, f0, f1))
        assert d is None, "step %d world %d contacts: %s" % (step, k, d)


def test_batch_equals_worlds_stepped_one_at_a_time():
    g = U.gpu()
    seeds = list(range(1, 33))
    solo = _worlds(g, seeds)
    src = _worlds(g, seeds)
    batch = _batch(g, src)
    try:
        assert g.m3d_gpu_batch_world_count(batch) == len(seeds)
        for step in range(60):
            for s in solo:
                s.step_only()
            g.m3d_world_step(batch, 1.0 / 60.0, 4)
            assert g.m3d_gpu_status(batch) == 0, g.m3d_gpu_last_error_string(batch)
            _compare(g, g, batch, solo, step)
    finally:
        g.m3d_world_destroy(batch)
        for s in solo + src:
            s.close()


def test_batch_through_sleep_equals_worlds_one_at_a_time():
    # long enough for worlds to fall asleep at different steps: each world's
    # stable tier is rebuilt on its own schedule
    g = U.gpu()
    seeds = [101, 102, 103, 104, 105, 106]
    solo = _worlds(g, seeds, a=24, b=1)
    src = _worlds(g, seeds, a=24, b=1)
    batch = _batch(g, src)
    try:
        slept = set()
        for step in range(300):
            for s in solo:
                s.step_only()
            g.m3d_world_step(batch, 1.0 / 60.0, 4)
            if step % 10 == 9 or step == 299:
                _compare(g, g, batch, solo, step)
                for k, s in enumerate(solo):
                    if g.m3d_world_profile(s.world).awakeBodyCount < 24:
                        slept.add(k)
        assert len(slept) >= 2, "bodies fell asleep in %d worlds: the stable-tier schedules were not exercised" % len(slept)
    finally:
        g.m3d_world_destroy(batch)
        for s in solo + src:
            s.close()


def test_batch_matches_the_reference():
    # 64 worlds of the batched-worlds workload (16-512 bodies, 0-4 ball or
    # hinge joints each) against the reference stepping each world alone,
    # 60 steps, every world compared after every step
    g, ref = U.gpu(), U.oracle_cr()
    seeds = list(range(7, 7 + 64))
    refs = _worlds(ref, seeds)
    src = _worlds(g, seeds)
    batch = _batch(g, src)
    try:
        for step in range(60):
            for s in refs:
                s.step_only()
            g.m3d_world_step(batch, 1.0 / 60.0, 4)
            _compare(g, ref, batch, refs, step)
    finally:
        g.m3d_world_destroy(batch)
        for s in refs + src:
            s.close()


def test_batch_refuses_what_it_cannot_do():
    g = U.gpu()
    src = _worlds(g, [1, 2])
    batch = _batch(g, src)
    try:
        from melon3d_b200 import api
        bd = g.m3d_body_def_default()
        sd = g.m3d_shape_def_default()
        assert g.m3d_body_create(batch, C.byref(bd), C.byref(sd)).index == -1
        r = g.m3d_world_ray_cast(batch, api.Vec3(0, 20, 0), api.Vec3(0, -40, 0))
        assert not r.hit
        g.m3d_world_step(src[0].world, 1.0 / 60.0, 4)
        arr = (C.c_void_p * 2)(src[0].world, src[1].world)
        assert not g.m3d_gpu_batch_create(arr, 2)  # a stepped world cannot join a batch
    finally:
        g.m3d_world_destroy(batch)
        for s in src:
            s.close()
