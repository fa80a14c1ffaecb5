"""Shared test helpers: the oracle loader (test infrastructure only), world
snapshots as numpy arrays, and lockstep comparison of two worlds."""
import ctypes as C
import os

import numpy as np
import pytest

from melon3d_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle", "_ref")
ORACLE_LIB = os.path.join(ORACLE_DIR, "libmelon3d_ref.so")

_libs = {}


def _load(name):
    if name not in _libs:
        path = os.path.join(ORACLE_DIR, name)
        if not os.path.exists(path):
            pytest.skip("oracle/_ref/%s not built (make -C oracle)" % name)
        _libs[name] = api.bind(C.CDLL(path))
    return _libs[name]


def oracle():
    """The reference library built from its own sources with contraction off
    (oracle/Makefile).  Skips the test when it has not been built."""
    return _load("libmelon3d_ref.so")


def oracle_cr():
    """Same, with libm's float sinf/cosf/atan2f evaluated in double and rounded
    once (oracle/cr_libm.h), as the GPU kernels do: the bit-level oracle for
    scenes in which bodies spin fast enough to reach those calls."""
    return _load("libmelon3d_ref_cr.so")


def oracle_fast():
    """The reference built with its own release flags (FMA contraction on)."""
    return _load("libmelon3d_ref_fast.so")


def gpu():
    return api.load_gpu()


def bodies(lib, world):
    n = lib.m3d_dbg_body_capacity(world)
    out = (api.DbgBody * max(n, 1))()
    lib.m3d_dbg_bodies(world, out, n)
    return np.ctypeslib.as_array(out)[:n].copy() if n else np.zeros(0, dtype=np.ctypeslib.as_array(out).dtype)


def contacts(lib, world):
    n = lib.m3d_dbg_contact_count(world)
    out = (api.DbgContact * max(n, 1))()
    lib.m3d_dbg_contacts(world, out, n)
    return np.ctypeslib.as_array(out)[:n].copy()


def island_labels(lib, world):
    n = lib.m3d_dbg_body_capacity(world)
    out = (C.c_int32 * max(n, 1))()
    lib.m3d_dbg_island_labels(world, out, n)
    return np.array(out[:n], dtype=np.int32)


def contact_colors(lib, world):
    n = lib.m3d_dbg_contact_count(world)
    out = (C.c_int32 * max(n, 1))()
    lib.m3d_dbg_contact_colors(world, out, n)
    return np.array(out[:n], dtype=np.int32)


def events(lib, world):
    """The world's current contact events, in list order: (begin, end), each
    an int64 array of rows (bodyA index, generation, bodyB index, generation,
    isSensor)."""
    ev = lib.m3d_world_contact_events(world)

    def rows(ptr, n):
        if n <= 0:
            return np.zeros((0, 5), np.int64)
        a = np.ctypeslib.as_array(ptr, shape=(n,))
        return np.stack([a["bodyA"]["index"], a["bodyA"]["generation"], a["bodyB"]["index"],
                         a["bodyB"]["generation"], a["isSensor"]], axis=1).astype(np.int64)
    return rows(ev.beginEvents, ev.beginCount), rows(ev.endEvents, ev.endCount)


def diff_events(er, eg):
    """First difference between two worlds' event lists (order included)."""
    for name, a, b in (("begin", er[0], eg[0]), ("end", er[1], eg[1])):
        if len(a) != len(b):
            return "%s events: %d vs %d" % (name, len(a), len(b))
        bad = np.nonzero((a != b).any(axis=1))[0]
        if len(bad):
            k = int(bad[0])
            return "%s event %d: %s vs %s" % (name, k, a[k].tolist(), b[k].tolist())
    return None


BODY_FIELDS = ("position", "rotation", "linearVelocity", "angularVelocity", "sleepTime", "smoothedEnergy",
               "isAwake", "inUse")
CONTACT_FIELDS = ("bodyA", "bodyB", "pointCount", "touching", "isSensor", "tunnelGuard", "normal", "friction",
                  "restitution", "rollingResistance")
POINT_FIELDS = ("localAnchorA", "localAnchorB", "frictionAnchorA", "frictionAnchorB", "separation", "id",
                "separationOffset", "slipDir")


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def diff_bodies(br, bg, live_only=True):
    """First mismatching (field, index) between two body snapshots, bitwise."""
    if len(br) != len(bg):
        return "body capacity %d vs %d" % (len(br), len(bg))
    for f in BODY_FIELDS:
        a, b = bits(br[f]), bits(bg[f])
        if live_only:
            m = br["inUse"] != 0
            a, b = a[m], b[m]
        if not np.array_equal(a, b):
            idx = np.nonzero((a != b).reshape(len(a), -1).any(axis=1))[0]
            return "body field %s differs at %d bodies (first live index %d)" % (f, len(idx), int(idx[0]))
    return None


def diff_contacts(cr, cg):
    if len(cr) != len(cg):
        return "contact count %d vs %d" % (len(cr), len(cg))
    for f in CONTACT_FIELDS:
        a, b = bits(cr[f]), bits(cg[f])
        if not np.array_equal(a, b):
            idx = np.nonzero((a != b).reshape(len(a), -1).any(axis=1))[0]
            return "contact field %s differs at %d contacts (first %d)" % (f, len(idx), int(idx[0]))
    pc = cr["pointCount"]
    for p in range(4):
        m = pc > p
        for f in POINT_FIELDS:
            a, b = bits(cr["points"][f][:, p][m]), bits(cg["points"][f][:, p][m])
            if not np.array_equal(a, b):
                idx = np.nonzero(m)[0][np.nonzero((a != b).reshape(len(a), -1).any(axis=1))[0]]
                return "point %d field %s differs at %d contacts (first %d)" % (p, f, len(idx), int(idx[0]))
    return None


def pose_error(br, bg):
    """max |dx| and max |dq| over live bodies (metres / quaternion units)."""
    m = br["inUse"] != 0
    dx = np.abs(br["position"][m].astype(np.float64) - bg["position"][m].astype(np.float64)).max(initial=0.0)
    qa, qb = br["rotation"][m].astype(np.float64), bg["rotation"][m].astype(np.float64)
    dq = np.minimum(np.abs(qa - qb).max(axis=1, initial=0.0), np.abs(qa + qb).max(axis=1, initial=0.0))
    return float(dx), float(dq.max(initial=0.0))
