"""The drop-in boundary: the GPU library exports every function the public
headers declare, loads without a GPU, and refuses to create a world when no
CUDA device exists (no silent CPU fallback)."""
import ctypes as C
import os
import re
import subprocess

import pytest

from melon3d_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"M3D_API\s+[\w\s\*]+?\b(m3d_\w+)\s*\(", text)))


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


def test_headers_declare_the_reference_api():
    names = declared("melon3d.h")
    # the reference's public header declares 49 functions (include/melon3d.h:452-527)
    assert len(names) == 49, names
    assert set(names) <= set(api.API_SYMBOLS)


def test_library_exports_every_declared_symbol():
    if not os.path.exists(api.GPU_LIB):
        pytest.skip("library not built")
    ex = exported(api.GPU_LIB)
    missing = [n for n in declared("melon3d.h") + declared("melon3d_gpu.h") if n not in ex]
    assert not missing, missing


def test_library_loads_and_binds_without_a_gpu():
    if not os.path.exists(api.GPU_LIB):
        pytest.skip("library not built")
    lib = api.bind(C.CDLL(api.GPU_LIB), gpu=True)
    d = lib.m3d_world_def_default()
    assert abs(d.gravity.y + 9.81) < 1e-6 and d.positionIterations == 2 and abs(d.gridCellSize - 1.5) < 1e-7
    s = lib.m3d_shape_def_default()
    assert s.type == api.SHAPE_SPHERE and abs(s.rollingResistance - 0.02) < 1e-9
    b = lib.m3d_body_def_default()
    assert b.type == api.BODY_STATIC and b.isAwake and abs(b.angularDamping - 0.05) < 1e-9


def test_no_world_without_cuda_device():
    if not os.path.exists(api.GPU_LIB):
        pytest.skip("library not built")
    probe = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True) if os.path.exists(
        "/usr/bin/nvidia-smi") else None
    if probe is not None and probe.returncode == 0 and "GPU" in probe.stdout:
        pytest.skip("a GPU is present")
    lib = api.bind(C.CDLL(api.GPU_LIB), gpu=True)
    d = lib.m3d_world_def_default()
    assert not lib.m3d_world_create(C.byref(d))


def test_struct_layouts_match_c():
    # sizes of the ABI structs as the C compiler lays them out
    src = r"""
#include "melon3d.h"
#include "melon3d_debug.h"
#include <stdio.h>
int main(void){printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(m3d_shape_def), sizeof(m3d_body_def),
 sizeof(m3d_world_def), sizeof(m3d_hinge_joint_def), sizeof(m3d_contact_event), sizeof(m3d_ray_result),
 sizeof(m3d_profile), sizeof(m3d_dbg_contact), sizeof(m3d_dbg_body), sizeof(m3d_distance_joint_def));return 0;}
"""
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = [int(x) for x in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    want = [C.sizeof(t) for t in (api.ShapeDef, api.BodyDef, api.WorldDef, api.HingeJointDef, api.ContactEvent,
                                  api.RayResult, api.Profile, api.DbgContact, api.DbgBody, api.DistanceJointDef)]
    assert got == want
