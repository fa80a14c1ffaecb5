"""Online autotuning of the serial-island kernel choice (m3d_gpu_autotune,
include/melon3d_gpu.h): the trials run on a batch's own steps and must not
change its results; the choice lands in the cache file and a later batch
picks it up at once."""
import ctypes as C
import os

import pytest

from melon3d_b200 import api, harness

from . import _util as U

pytestmark = pytest.mark.gpu


def _batch(g, seeds):
    scenes = [harness.Scene(g, harness.BATCH_WORLD, s) for s in seeds]
    arr = (C.c_void_p * len(scenes))(*[s.world for s in scenes])
    b = g.m3d_gpu_batch_create(arr, len(scenes))
    for s in scenes:
        s.close()
    assert b
    return b


def test_trials_leave_the_results_unchanged_and_the_choice_is_cached(tmp_path, monkeypatch):
    cache = str(tmp_path / "autotune.txt")
    monkeypatch.setenv("M3D_AUTOTUNE_CACHE", cache)
    g = U.gpu()
    seeds = list(range(200, 248))
    tuned, plain = _batch(g, seeds), _batch(g, seeds)
    try:
        assert g.m3d_gpu_autotune(tuned, 2) == 0  # nothing cached yet: trials start
        tc, tm = C.c_int32(), C.c_int32()
        assert g.m3d_gpu_autotune_state(tuned, C.byref(tc), C.byref(tm)) == 1
        for step in range(30):  # 6 candidates x 2 steps x 2 rounds, then the choice
            g.m3d_world_step(tuned, 1.0 / 60.0, 4)
            g.m3d_world_step(plain, 1.0 / 60.0, 4)
            d = U.diff_bodies(U.bodies(g, plain), U.bodies(g, tuned))
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_contacts(U.contacts(g, plain), U.contacts(g, tuned))
            assert d is None, "step %d: %s" % (step, d)
        assert g.m3d_gpu_autotune_state(tuned, C.byref(tc), C.byref(tm)) == 2
        assert os.path.exists(cache) and open(cache).read().count("\n") == 1
        again = _batch(g, seeds)
        try:
            assert g.m3d_gpu_autotune(again, 2) == 1  # found in the cache
            c2, m2 = C.c_int32(), C.c_int32()
            assert g.m3d_gpu_autotune_state(again, C.byref(c2), C.byref(m2)) == 2
            assert (c2.value, m2.value) == (tc.value, tm.value)
        finally:
            g.m3d_world_destroy(again)
        assert g.m3d_gpu_status(tuned) == api.GPU_OK
    finally:
        g.m3d_world_destroy(tuned)
        g.m3d_world_destroy(plain)
