"""m3d_gpu_sphere_cast_noalloc (include/melon3d_gpu.h): the sphere cast over a
fixed device scratch block built into the library, against the allocating
m3d_world_sphere_cast on the same world.  Both run the same kernels in the
same order, so the results must agree exactly (the bit-exact bar of the other
GPU tests).  Collected last so that it also runs after every other test in the
same process, when the block has already been set up and used."""
import ctypes as C

import numpy as np
import pytest

from melon3d_b200 import api
from melon3d_b200 import harness

pytestmark = pytest.mark.gpu


def _lib():
    return api.load_gpu()


def _fields(r):
    return (r.hit, r.body.index, r.body.generation, np.float32(r.fraction).tobytes(),
            np.array([r.point.x, r.point.y, r.point.z], np.float32).tobytes(),
            np.array([r.normal.x, r.normal.y, r.normal.z], np.float32).tobytes())


def _casts(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        x, z = rng.uniform(-45.0, 45.0, 2)
        if k % 4 == 3:
            # upward from just above the ground: mostly misses or starts inside
            origin, trans = (x, 0.2, z), (0.0, 20.0, 0.0)
        else:
            origin, trans = (x, 70.0, z), (rng.uniform(-5, 5), -80.0, rng.uniform(-5, 5))
        radius = float(rng.uniform(0.05, 1.5))
        mask = 0xFFFFFFFF if k % 5 else 0x1
        out.append((api.Vec3(*map(float, origin)), radius, api.Vec3(*map(float, trans)), mask))
    return out


def _noalloc(lib, world, cast):
    r = api.RayResult()
    rc = lib.m3d_gpu_sphere_cast_noalloc(world, cast[0], cast[1], cast[2], cast[3], C.byref(r))
    return rc, r


def _scene(bodies, steps):
    lib = _lib()
    scene = harness.Scene(lib, harness.RAIN, 5, bodies, 0)
    if steps:
        scene.run(steps)
    return lib, scene


def test_two_calls_in_a_row_match_the_allocating_cast():
    lib, scene = _scene(3000, 30)
    try:
        world = scene.world
        hits = 0
        casts = _casts(11, 48)
        for a, b in zip(casts[0::2], casts[1::2]):
            rc_a, ra = _noalloc(lib, world, a)
            rc_b, rb = _noalloc(lib, world, b)
            assert rc_a == api.GPU_OK and rc_b == api.GPU_OK
            ea = lib.m3d_world_sphere_cast(world, *a)
            eb = lib.m3d_world_sphere_cast(world, *b)
            assert _fields(ra) == _fields(ea)
            assert _fields(rb) == _fields(eb)
            hits += ea.hit + eb.hit
        assert 0 < hits < len(casts)
        assert lib.m3d_gpu_status(world) == api.GPU_OK
    finally:
        scene.close()


def test_hit_then_miss_leaves_no_stale_result():
    lib, scene = _scene(2000, 20)
    try:
        world = scene.world
        down = (api.Vec3(0.0, 70.0, 0.0), 60.0, api.Vec3(0.0, -80.0, 0.0), 0xFFFFFFFF)
        away = (api.Vec3(0.0, 500.0, 0.0), 0.5, api.Vec3(0.0, 10.0, 0.0), 0xFFFFFFFF)
        rc1, r1 = _noalloc(lib, world, down)
        rc2, r2 = _noalloc(lib, world, away)
        assert rc1 == api.GPU_OK and rc2 == api.GPU_OK
        assert r1.hit and not r2.hit and r2.body.index == -1
        assert _fields(r1) == _fields(lib.m3d_world_sphere_cast(world, *down))
        assert _fields(r2) == _fields(lib.m3d_world_sphere_cast(world, *away))
    finally:
        scene.close()


def test_pending_edits_are_rejected_until_uploaded():
    lib, scene = _scene(500, 5)
    try:
        world = scene.world
        bd = lib.m3d_body_def_default()
        bd.type = api.BODY_DYNAMIC
        bd.position = api.Vec3(0.0, 80.0, 0.0)
        sd = lib.m3d_shape_def_default()
        sd.radius = 2.0
        lib.m3d_body_create(world, C.byref(bd), C.byref(sd))
        cast = (api.Vec3(0.0, 90.0, 0.0), 0.5, api.Vec3(0.0, -20.0, 0.0), 0xFFFFFFFF)
        rc, r = _noalloc(lib, world, cast)
        assert rc == api.GPU_ERR_PENDING and not r.hit
        e = lib.m3d_world_sphere_cast(world, *cast)  # uploads the new body
        rc, r = _noalloc(lib, world, cast)
        assert rc == api.GPU_OK and e.hit and _fields(r) == _fields(e)
    finally:
        scene.close()


def test_worlds_beyond_the_limit_are_rejected():
    lib, scene = _scene(65537, 0)
    try:
        assert lib.m3d_gpu_body_capacity(scene.world) > 65536
        cast = (api.Vec3(0.0, 70.0, 0.0), 0.5, api.Vec3(0.0, -80.0, 0.0), 0xFFFFFFFF)
        rc, r = _noalloc(lib, scene.world, cast)
        assert rc == api.GPU_ERR_LIMIT and not r.hit
        assert lib.m3d_gpu_sphere_cast_noalloc(scene.world, cast[0], cast[1], cast[2], cast[3], None) == \
            api.GPU_ERR_ARGUMENT
    finally:
        scene.close()


def test_calls_allocate_no_device_memory():
    """The defining property: on a warm world, a run of fixed-scratch casts
    makes no device allocation (the library's cudaMalloc counter and the
    device's free memory are unchanged), while the results still match the
    allocating cast, which is made after the run."""
    import torch
    lib, scene = _scene(3000, 10)
    try:
        world = scene.world
        casts = _casts(23, 16)
        _noalloc(lib, world, casts[0])  # the first call on the device sets up the scratch address
        torch.cuda.synchronize()
        allocs = lib.m3d_gpu_profiler_allocations()
        free0, _ = torch.cuda.mem_get_info()
        got = [_noalloc(lib, world, c) for c in casts]
        torch.cuda.synchronize()
        assert lib.m3d_gpu_profiler_allocations() == allocs
        assert torch.cuda.mem_get_info()[0] == free0
        for c, (rc, r) in zip(casts, got):
            assert rc == api.GPU_OK
            assert _fields(r) == _fields(lib.m3d_world_sphere_cast(world, *c))
    finally:
        scene.close()


def test_largest_accepted_world():
    # exactly 65536 body slots (the ground and 65535 rain bodies): accepted
    lib, scene = _scene(65535, 2)
    try:
        world = scene.world
        assert lib.m3d_gpu_body_capacity(world) == 65536
        for c in _casts(31, 6):
            rc, r = _noalloc(lib, world, c)
            assert rc == api.GPU_OK
            assert _fields(r) == _fields(lib.m3d_world_sphere_cast(world, *c))
    finally:
        scene.close()
