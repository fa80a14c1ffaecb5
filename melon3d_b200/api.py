"""ctypes binding of Melon3D's C API (include/melon3d.h) and of the GPU
extensions (include/melon3d_gpu.h, include/melon3d_debug.h).

`bind(cdll)` attaches argument/result types to any shared library that
exports the Melon3D C API, so the same Python scene code drives the GPU
library (`load_gpu()`).  Structures mirror the C layouts field for field.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
GPU_LIB = os.path.join(HERE, "lib", "libmelon3d_gpu.so")

BODY_STATIC, BODY_KINEMATIC, BODY_DYNAMIC = 0, 1, 2
SHAPE_SPHERE, SHAPE_CAPSULE, SHAPE_BOX = 0, 1, 2
PI = 3.14159265358979323846


class Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]

    def tup(self):
        return (self.x, self.y, self.z)


class Quat(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]

    def tup(self):
        return (self.x, self.y, self.z, self.w)


class Transform(C.Structure):
    _fields_ = [("p", Vec3), ("q", Quat)]


class AABB(C.Structure):
    _fields_ = [("lowerBound", Vec3), ("upperBound", Vec3)]


class BodyId(C.Structure):
    _fields_ = [("index", C.c_int32), ("generation", C.c_uint32)]


class JointId(C.Structure):
    _fields_ = [("index", C.c_int32), ("generation", C.c_uint32)]


class Filter(C.Structure):
    _fields_ = [("categoryBits", C.c_uint32), ("maskBits", C.c_uint32), ("groupIndex", C.c_int32)]


class ShapeDef(C.Structure):
    _fields_ = [("type", C.c_int), ("radius", C.c_float), ("halfHeight", C.c_float), ("halfExtents", Vec3),
                ("density", C.c_float), ("friction", C.c_float), ("restitution", C.c_float),
                ("rollingResistance", C.c_float), ("filter", Filter), ("isSensor", C.c_bool)]


class BodyDef(C.Structure):
    _fields_ = [("type", C.c_int), ("position", Vec3), ("orientation", Quat), ("linearVelocity", Vec3),
                ("angularVelocity", Vec3), ("linearDamping", C.c_float), ("angularDamping", C.c_float),
                ("gravityScale", C.c_float), ("enableSleep", C.c_bool), ("isAwake", C.c_bool),
                ("userData", C.c_uint64)]


class WorldDef(C.Structure):
    _fields_ = [("gravity", Vec3), ("workerCount", C.c_int32), ("positionIterations", C.c_int32),
                ("gridCellSize", C.c_float), ("enableSleep", C.c_bool)]


class DistanceJointDef(C.Structure):
    _fields_ = [("bodyA", BodyId), ("bodyB", BodyId), ("localAnchorA", Vec3), ("localAnchorB", Vec3),
                ("length", C.c_float), ("hertz", C.c_float), ("dampingRatio", C.c_float)]


class BallJointDef(C.Structure):
    _fields_ = [("bodyA", BodyId), ("bodyB", BodyId), ("localAnchorA", Vec3), ("localAnchorB", Vec3)]


class HingeJointDef(C.Structure):
    _fields_ = [("bodyA", BodyId), ("bodyB", BodyId), ("localAnchorA", Vec3), ("localAnchorB", Vec3),
                ("localAxisA", Vec3), ("localAxisB", Vec3), ("enableLimit", C.c_bool), ("lowerAngle", C.c_float),
                ("upperAngle", C.c_float), ("enableMotor", C.c_bool), ("motorSpeed", C.c_float),
                ("maxMotorTorque", C.c_float)]


class WeldJointDef(C.Structure):
    _fields_ = [("bodyA", BodyId), ("bodyB", BodyId), ("localAnchorA", Vec3), ("localAnchorB", Vec3)]


class ContactEvent(C.Structure):
    _fields_ = [("bodyA", BodyId), ("bodyB", BodyId), ("isSensor", C.c_bool)]


class ContactEvents(C.Structure):
    _fields_ = [("beginEvents", C.POINTER(ContactEvent)), ("beginCount", C.c_int32),
                ("endEvents", C.POINTER(ContactEvent)), ("endCount", C.c_int32)]


class RayResult(C.Structure):
    _fields_ = [("body", BodyId), ("point", Vec3), ("normal", Vec3), ("fraction", C.c_float), ("hit", C.c_bool)]


class Profile(C.Structure):
    _fields_ = [("stepMs", C.c_float), ("broadphaseMs", C.c_float), ("narrowphaseMs", C.c_float),
                ("solverMs", C.c_float), ("bodyCount", C.c_int32), ("awakeBodyCount", C.c_int32),
                ("contactCount", C.c_int32), ("touchingContactCount", C.c_int32), ("islandCount", C.c_int32)]


class DbgPoint(C.Structure):
    _fields_ = [("localAnchorA", C.c_float * 3), ("localAnchorB", C.c_float * 3),
                ("frictionAnchorA", C.c_float * 3), ("frictionAnchorB", C.c_float * 3),
                ("separation", C.c_float), ("id", C.c_uint32), ("lambdaN", C.c_float), ("lambdaT", C.c_float),
                ("separationOffset", C.c_float), ("slipDir", C.c_float * 3)]


class DbgContact(C.Structure):
    _fields_ = [("bodyA", C.c_int32), ("bodyB", C.c_int32), ("pointCount", C.c_int32), ("touching", C.c_uint8),
                ("isSensor", C.c_uint8), ("tunnelGuard", C.c_uint8), ("hasCache", C.c_uint8),
                ("normal", C.c_float * 3), ("friction", C.c_float), ("restitution", C.c_float),
                ("rollingResistance", C.c_float), ("points", DbgPoint * 4)]


class DbgBody(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("rotation", C.c_float * 4), ("linearVelocity", C.c_float * 3),
                ("angularVelocity", C.c_float * 3), ("prevPosition", C.c_float * 3), ("prevRotation", C.c_float * 4),
                ("invInertiaWorld", C.c_float * 9), ("sleepTime", C.c_float), ("smoothedEnergy", C.c_float),
                ("fatLower", C.c_float * 3), ("fatUpper", C.c_float * 3), ("hasFatAABB", C.c_uint8),
                ("isAwake", C.c_uint8), ("inUse", C.c_uint8), ("pad", C.c_uint8)]


OverlapFn = C.CFUNCTYPE(C.c_bool, BodyId, C.c_void_p)

W = C.c_void_p

_PROTOS = {
    "m3d_world_def_default": (WorldDef, []),
    "m3d_body_def_default": (BodyDef, []),
    "m3d_shape_def_default": (ShapeDef, []),
    "m3d_hinge_joint_def_default": (HingeJointDef, []),
    "m3d_weld_joint_def_default": (WeldJointDef, []),
    "m3d_world_create": (W, [C.POINTER(WorldDef)]),
    "m3d_world_destroy": (None, [W]),
    "m3d_world_step": (None, [W, C.c_float, C.c_int]),
    "m3d_body_create": (BodyId, [W, C.POINTER(BodyDef), C.POINTER(ShapeDef)]),
    "m3d_body_destroy": (None, [W, BodyId]),
    "m3d_body_is_valid": (C.c_bool, [W, BodyId]),
    "m3d_body_position": (Vec3, [W, BodyId]),
    "m3d_body_rotation": (Quat, [W, BodyId]),
    "m3d_body_transform": (Transform, [W, BodyId]),
    "m3d_body_set_transform": (None, [W, BodyId, Vec3, Quat]),
    "m3d_body_linear_velocity": (Vec3, [W, BodyId]),
    "m3d_body_angular_velocity": (Vec3, [W, BodyId]),
    "m3d_body_set_linear_velocity": (None, [W, BodyId, Vec3]),
    "m3d_body_set_angular_velocity": (None, [W, BodyId, Vec3]),
    "m3d_body_apply_impulse": (None, [W, BodyId, Vec3, Vec3]),
    "m3d_body_apply_force": (None, [W, BodyId, Vec3]),
    "m3d_body_apply_force_at_point": (None, [W, BodyId, Vec3, Vec3]),
    "m3d_body_apply_torque": (None, [W, BodyId, Vec3]),
    "m3d_body_apply_angular_impulse": (None, [W, BodyId, Vec3]),
    "m3d_body_mass": (C.c_float, [W, BodyId]),
    "m3d_body_get_type": (C.c_int, [W, BodyId]),
    "m3d_body_is_awake": (C.c_bool, [W, BodyId]),
    "m3d_body_wake": (None, [W, BodyId]),
    "m3d_body_user_data": (C.c_uint64, [W, BodyId]),
    "m3d_body_set_user_data": (None, [W, BodyId, C.c_uint64]),
    "m3d_body_friction": (C.c_float, [W, BodyId]),
    "m3d_body_set_friction": (None, [W, BodyId, C.c_float]),
    "m3d_body_restitution": (C.c_float, [W, BodyId]),
    "m3d_body_set_restitution": (None, [W, BodyId, C.c_float]),
    "m3d_world_gravity": (Vec3, [W]),
    "m3d_world_set_gravity": (None, [W, Vec3]),
    "m3d_joint_create_distance": (JointId, [W, C.POINTER(DistanceJointDef)]),
    "m3d_joint_create_ball": (JointId, [W, C.POINTER(BallJointDef)]),
    "m3d_joint_create_hinge": (JointId, [W, C.POINTER(HingeJointDef)]),
    "m3d_joint_create_weld": (JointId, [W, C.POINTER(WeldJointDef)]),
    "m3d_joint_destroy": (None, [W, JointId]),
    "m3d_joint_hinge_angle": (C.c_float, [W, JointId]),
    "m3d_joint_hinge_set_motor": (None, [W, JointId, C.c_bool, C.c_float, C.c_float]),
    "m3d_world_ray_cast": (RayResult, [W, Vec3, Vec3]),
    "m3d_world_ray_cast_filtered": (RayResult, [W, Vec3, Vec3, C.c_uint32]),
    "m3d_world_sphere_cast": (RayResult, [W, Vec3, C.c_float, Vec3, C.c_uint32]),
    "m3d_world_overlap_aabb": (None, [W, AABB, OverlapFn, C.c_void_p]),
    "m3d_world_contact_events": (ContactEvents, [W]),
    "m3d_world_profile": (Profile, [W]),
    # snapshot records (both the GPU library and the test oracle export these)
    "m3d_dbg_body_capacity": (C.c_int32, [W]),
    "m3d_dbg_bodies": (None, [W, C.POINTER(DbgBody), C.c_int32]),
    "m3d_dbg_contact_count": (C.c_int32, [W]),
    "m3d_dbg_contacts": (None, [W, C.POINTER(DbgContact), C.c_int32]),
    "m3d_dbg_island_labels": (None, [W, C.POINTER(C.c_int32), C.c_int32]),
    "m3d_dbg_contact_colors": (None, [W, C.POINTER(C.c_int32), C.c_int32]),
}

_GPU_PROTOS = {
    "m3d_gpu_body_capacity": (C.c_int32, [W]),
    "m3d_gpu_read_poses": (None, [W, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32]),
    "m3d_gpu_last_step_device_ms": (C.c_float, [W]),
    "m3d_gpu_status": (C.c_int32, [W]),
    "m3d_gpu_set_giant_island_contacts": (None, [W, C.c_int32]),
    "m3d_gpu_set_wait_limit": (None, [W, C.c_int64]),
    "m3d_gpu_fast_path_steps": (C.c_int64, [W]),
    "m3d_gpu_autotune": (C.c_int32, [W, C.c_int32]),
    "m3d_gpu_autotune_state": (C.c_int32, [W, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "m3d_gpu_clear_status": (None, [W]),
    "m3d_gpu_giant_profile": (C.c_int32, [W, C.POINTER(C.c_double), C.c_int32]),
    "m3d_gpu_batch_create": (W, [C.POINTER(W), C.c_int32]),
    "m3d_gpu_batch_world_count": (C.c_int32, [W]),
    "m3d_gpu_batch_first_body": (C.c_int32, [W, C.c_int32]),
    "m3d_gpu_last_error_string": (C.c_char_p, [W]),
    "m3d_gpu_step_counters": (C.c_int32, [W, C.POINTER(C.c_uint32), C.c_int32]),
    "m3d_gpu_profiler_reset": (None, [C.c_char_p]),
    "m3d_gpu_profiler_launches": (C.c_longlong, []),
    "m3d_gpu_profiler_allocations": (C.c_longlong, []),
    "m3d_gpu_profiler_kernel": (None, [C.POINTER(C.c_float), C.POINTER(C.c_int32)]),
    "m3d_gpu_profiler_bytes": (None, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "m3d_gpu_profiler_table": (C.c_int32, [C.c_char_p, C.c_int32]),
    "m3d_gpu_sphere_cast_noalloc": (C.c_int32, [W, Vec3, C.c_float, Vec3, C.c_uint32, C.POINTER(RayResult)]),
    "m3d_gpu_tape_begin": (C.c_int32, [W, C.c_int32]),
    "m3d_gpu_tape_end": (None, [W]),
    "m3d_gpu_tape_steps": (C.c_int32, [W]),
    "m3d_gpu_tape_bytes": (C.c_int64, [W]),
    "m3d_gpu_tape_warp_islands": (C.c_int64, [W]),
    "m3d_gpu_tape_supported": (C.c_int32, [W, C.c_char_p, C.c_int32]),
    "m3d_gpu_tape_replay": (C.c_int32, [W] + [C.POINTER(C.c_float)] * 4 + [C.c_int32]),
    "m3d_gpu_step_backward": (C.c_int32, [W] + [C.POINTER(C.c_float)] * 11 + [C.c_int32]),
    "m3d_gpu_step_backward_fp64_host": (C.c_int32, [W] + [C.POINTER(C.c_double)] * 11 + [C.c_int32]),
    "m3d_gpu_tape_regenerate_host": (C.c_int32, [W, C.c_int32] + [C.POINTER(C.c_double)] * 9 + [C.c_int32]),
}

# status codes of melon3d_gpu.h
GPU_OK = 0
GPU_ERR_CUDA = -1
GPU_ERR_ALLOC = -2
GPU_ERR_HASH = -3
GPU_ERR_LIMIT = -4
GPU_ERR_PENDING = -5
GPU_ERR_ARGUMENT = -6
GPU_ERR_WAIT = -7
GPU_ERR_UNSUPPORTED = -8

API_SYMBOLS = sorted(_PROTOS)
GPU_SYMBOLS = sorted(_GPU_PROTOS)


def bind(lib, gpu=False):
    """Attach prototypes of the C API (and the GPU extensions) to a CDLL."""
    protos = dict(_PROTOS)
    if gpu:
        protos.update(_GPU_PROTOS)
    for name, (res, args) in protos.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_gpu = None


def load_gpu():
    """The GPU library.  Raises when it is missing: there is no CPU fallback."""
    global _gpu
    if _gpu is None:
        if not os.path.exists(GPU_LIB):
            raise RuntimeError("libmelon3d_gpu.so is not built (python -m melon3d_b200.build)")
        _gpu = bind(C.CDLL(GPU_LIB), gpu=True)
    return _gpu


def v3(x, y, z):
    return Vec3(x, y, z)


def quat_axis_angle(lib_unused, axis, angle):
    """m3d_quat_axis_angle with libm sinf/cosf, as the inline helper computes it."""
    import math
    import numpy as np
    ax = np.array(axis, dtype=np.float32)
    n = float(np.sqrt(np.float32(ax[0] * ax[0] + ax[1] * ax[1]) + np.float32(ax[2] * ax[2])))
    f = np.float32
    if n < 1e-12:
        nx = ny = nz = f(0)
    else:
        inv = f(1.0) / f(n)
        nx, ny, nz = f(inv * ax[0]), f(inv * ax[1]), f(inv * ax[2])
    half = f(f(0.5) * f(angle))
    s = f(math.sin(half))
    return Quat(f(s * nx), f(s * ny), f(s * nz), f(math.cos(half)))
