"""Reverse functions of the differentiable substep (m3d_diff.h) against
central finite differences, in double precision on the CPU: integration,
contact preparation, normal projection, stiction friction, velocity
reconstruction and the velocity pass, each on random inputs (both branches of
the rotation update and of the log map, static and dynamic partners, budgets
that take either side of the friction caps)."""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "diff", "diff_ops_check.cpp")
INC = os.path.join(ROOT, "melon3d_b200", "csrc")

_lib = None


def lib():
    global _lib
    if _lib is None:
        d = tempfile.mkdtemp(prefix="m3d_diffcheck_")
        so = os.path.join(d, "diffcheck.so")
        subprocess.run(["g++", "-std=c++17", "-O1", "-fPIC", "-shared", "-I" + INC, SRC, "-o", so], check=True)
        _lib = C.CDLL(so)
        for name in ("check_integrate", "check_prepare", "check_normals", "check_friction", "check_reconstruct",
                     "check_velocity", "check_prepare_contact", "check_normals_contact", "check_friction_contact",
                     "check_velocity_contact", "check_generation"):
            f = getattr(_lib, name)
            f.restype = C.c_double
            f.argtypes = [C.c_uint64]
    return _lib


@pytest.mark.parametrize("op", ["integrate", "prepare", "normals", "friction", "reconstruct", "velocity"])
def test_reverse_matches_finite_differences(op):
    f = getattr(lib(), "check_" + op)
    worst = max(f(seed) for seed in range(1, 41))
    assert worst < 1e-5, "%s: worst relative error %.3g" % (op, worst)


@pytest.mark.parametrize("op", ["prepare", "normals", "friction", "velocity"])
def test_manifold_adjoints_match_finite_differences(op):
    """Adjoints of the manifold data each operation reads (normal, local and
    stiction anchors, separation offsets)."""
    f = getattr(lib(), "check_%s_contact" % op)
    worst = max(f(seed) for seed in range(1, 41))
    assert worst < 1e-5, "%s: worst relative error %.3g" % (op, worst)


def test_generation_jacobian_matches_finite_differences():
    """Dual-number derivatives of a generated manifold (box-box face and edge
    contacts, sphere-box both ways, sphere-sphere) with respect to the two
    poses, against central differences of the same generation in double."""
    worst = max(lib().check_generation(seed) for seed in range(1, 51))
    assert worst < 1e-5, "worst relative error %.3g" % worst
