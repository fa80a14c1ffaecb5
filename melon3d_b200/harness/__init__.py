"""Seeded benchmark scenes (harness/scenes.cpp) driven through the C API of a
bound library (see melon3d_b200.api.bind)."""
import ctypes as C
import os
import subprocess

from .. import api

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SRC = os.path.join(HERE, "scenes.cpp")
LIB = os.path.join(os.path.dirname(HERE), "lib", "libm3d_scenes.so")

PYRAMID, RAIN, PILE, RAFT, BATCH_WORLD, INCLINE, JOINTED_RAFT, SETTLED_STACKS = 0, 1, 2, 3, 4, 5, 6, 7


class M3dApi(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in (
        "world_def_default", "body_def_default", "shape_def_default", "world_create", "world_destroy",
        "world_step", "body_create", "body_destroy", "body_position", "world_profile", "read_poses",
        "joint_create_ball", "joint_create_hinge", "hinge_joint_def_default", "joint_create_distance",
        "joint_create_weld", "weld_joint_def_default")]


def build(force=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
               "-I" + os.path.join(ROOT, "include"), SRC, "-o", LIB]
        subprocess.run(cmd, check=True)
    return LIB


_lib = None


def _load():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        _lib.scn_create.restype = C.c_void_p
        _lib.scn_create.argtypes = [C.POINTER(M3dApi), C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int]
        _lib.scn_world.restype = C.c_void_p
        _lib.scn_world.argtypes = [C.c_void_p]
        _lib.scn_dynamic_count.restype = C.c_int32
        _lib.scn_dynamic_count.argtypes = [C.c_void_p]
        _lib.scn_run.restype = C.c_int64
        _lib.scn_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]
        _lib.scn_dynamic_ids.restype = C.c_int32
        _lib.scn_dynamic_ids.argtypes = [C.c_void_p, C.POINTER(api.BodyId), C.c_int32]
        _lib.scn_churn.restype = None
        _lib.scn_churn.argtypes = [C.c_void_p]
        _lib.scn_step_only.restype = None
        _lib.scn_step_only.argtypes = [C.c_void_p, C.c_int]
        _lib.scn_batch_world_bodies.restype = C.c_int32
        _lib.scn_batch_world_bodies.argtypes = [C.c_uint64]
        _lib.scn_destroy.restype = None
        _lib.scn_destroy.argtypes = [C.c_void_p]
    return _lib


def api_table(lib):
    """Function-pointer table of a library exporting the Melon3D C API."""
    t = M3dApi()
    names = {"world_def_default": "m3d_world_def_default", "body_def_default": "m3d_body_def_default",
             "shape_def_default": "m3d_shape_def_default", "world_create": "m3d_world_create",
             "world_destroy": "m3d_world_destroy", "world_step": "m3d_world_step",
             "body_create": "m3d_body_create", "body_destroy": "m3d_body_destroy",
             "body_position": "m3d_body_position", "world_profile": "m3d_world_profile"}
    for field, sym in names.items():
        setattr(t, field, C.cast(getattr(lib, sym), C.c_void_p).value)
    if hasattr(lib, "m3d_gpu_read_poses"):
        t.read_poses = C.cast(lib.m3d_gpu_read_poses, C.c_void_p).value
    for field, sym in (("joint_create_ball", "m3d_joint_create_ball"), ("joint_create_hinge", "m3d_joint_create_hinge"),
                       ("hinge_joint_def_default", "m3d_hinge_joint_def_default"),
                       ("joint_create_distance", "m3d_joint_create_distance"),
                       ("joint_create_weld", "m3d_joint_create_weld"),
                       ("weld_joint_def_default", "m3d_weld_joint_def_default")):
        setattr(t, field, C.cast(getattr(lib, sym), C.c_void_p).value)
    return t


def batch_world_bodies(seed):
    """Dynamic bodies of world `seed` of the batched-worlds scene, without
    building it (same generator as the scene)."""
    return int(_load().scn_batch_world_bodies(seed))


class Scene:
    """A seeded scene in a world of `lib` (a library bound with api.bind)."""

    def __init__(self, lib, kind, seed=1, a=0, b=0, c=0, workers=0):
        self.lib = lib
        self.sl = _load()
        self.table = api_table(lib)
        self.handle = self.sl.scn_create(C.byref(self.table), kind, seed, a, b, c, workers)
        if not self.handle:
            raise RuntimeError("world creation failed")
        self.world = self.sl.scn_world(self.handle)

    def run(self, steps, substeps=4, per_step=False):
        wall = C.c_double(0.0)
        ms = (C.c_float * steps)() if per_step else None
        bs = self.sl.scn_run(self.handle, steps, substeps, C.byref(wall), ms)
        return bs, wall.value, (list(ms) if per_step else None)

    def churn(self):
        self.sl.scn_churn(self.handle)

    def step_only(self, substeps=4):
        self.sl.scn_step_only(self.handle, substeps)

    def dynamic_ids(self):
        n = self.sl.scn_dynamic_count(self.handle)
        out = (api.BodyId * max(n, 1))()
        self.sl.scn_dynamic_ids(self.handle, out, n)
        return [out[i] for i in range(n)]

    def close(self):
        if self.handle:
            self.sl.scn_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
