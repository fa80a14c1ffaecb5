"""Failure detection of the bounded device-side waits (include/melon3d_gpu.h,
m3d_gpu_set_wait_limit).  The waits are made to run out on purpose by a
limit of zero polls; nothing here faults, traps or hangs the GPU.

- a look-back scan that gives up raises M3D_GPU_ERR_WAIT and still computes
  the exact prefix, so the step's results stay bit-identical to a twin world
  whose scans never gave up;
- a whole-GPU island solve whose grid barrier gives up raises
  M3D_GPU_ERR_WAIT and stops at that barrier; the world keeps working: after
  the status is cleared and the default limits restored it steps on with
  status M3D_GPU_OK.
"""
import ctypes as C

import numpy as np
import pytest

from melon3d_b200 import api, harness

from . import _util as U

pytestmark = pytest.mark.gpu


def test_scan_that_gives_up_keeps_exact_results():
    g = U.gpu()
    a = harness.Scene(g, harness.RAIN, 2, 20000, 200)
    b = harness.Scene(g, harness.RAIN, 2, 20000, 200)
    try:
        a.run(3)
        b.run(3)
        assert g.m3d_gpu_status(b.world) == api.GPU_OK
        g.m3d_gpu_set_wait_limit(b.world, 0)  # no scan tile waits for its predecessors
        for step in range(5):
            a.run(1)
            b.run(1)
            assert g.m3d_gpu_status(a.world) == api.GPU_OK
            assert g.m3d_gpu_status(b.world) == api.GPU_ERR_WAIT
            d = U.diff_contacts(U.contacts(g, a.world), U.contacts(g, b.world))
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_bodies(U.bodies(g, a.world), U.bodies(g, b.world))
            assert d is None, "step %d: %s" % (step, d)
        assert b"wait" in g.m3d_gpu_last_error_string(b.world)
    finally:
        a.close()
        b.close()


def test_giant_solve_that_gives_up_stops_and_the_world_steps_on():
    g = U.gpu()
    s = harness.Scene(g, harness.PILE, 3, 20, 40, 20)  # one island of tens of thousands of contacts
    g.m3d_gpu_set_giant_island_contacts(s.world, 300)  # solved by the whole-GPU kernel
    try:
        s.run(2)
        assert g.m3d_gpu_status(s.world) == api.GPU_OK
        g.m3d_gpu_set_wait_limit(s.world, 0)
        s.run(1)
        assert g.m3d_gpu_status(s.world) == api.GPU_ERR_WAIT
        g.m3d_gpu_clear_status(s.world)
        g.m3d_gpu_set_wait_limit(s.world, -1)
        assert g.m3d_gpu_status(s.world) == api.GPU_OK
        for _ in range(5):
            s.run(1)
            assert g.m3d_gpu_status(s.world) == api.GPU_OK, g.m3d_gpu_last_error_string(s.world)
        cnt = (C.c_uint32 * 64)()
        g.m3d_gpu_step_counters(s.world, cnt, 64)
        assert cnt[28] == 1  # giantIslands: the whole-GPU kernel ran again
        b = U.bodies(g, s.world)
        live = b["inUse"] != 0
        assert np.isfinite(b["position"][live]).all() and np.isfinite(b["rotation"][live]).all()
    finally:
        s.close()
