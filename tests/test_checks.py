"""The reference's 52 closed-form / behavioural checks, run against the
oracle on the CPU (validates the restatement in checks52.py) and against the
GPU world on a B200."""
import pytest

from . import _util as U
from . import checks52

SCEN = [pytest.param(f, id=f.__name__) for f in checks52.SCENARIOS]


def test_check_count_is_52():
    assert checks52 is not None
    # counted by running every scenario on the oracle in test_oracle_checks
    assert len(checks52.SCENARIOS) == 23


@pytest.mark.parametrize("scenario", SCEN)
def test_oracle_checks(scenario):
    lib = U.oracle()
    results = scenario(lib)
    bad = [(name, val) for name, ok, val in results if not ok]
    assert not bad, bad


@pytest.mark.gpu
@pytest.mark.parametrize("scenario", SCEN)
def test_gpu_checks(scenario):
    lib = U.gpu()
    results = scenario(lib)
    bad = [(name, val) for name, ok, val in results if not ok]
    assert not bad, bad


def test_total_checks_52():
    lib = U.oracle()
    n = sum(len(f(lib)) for f in checks52.SCENARIOS)
    assert n == 52


@pytest.mark.gpu
def test_gpu_friction_laws_against_closed_form():
    """Coulomb sliding and rolling accelerations on the GPU world, at the
    reference test's integration (1/240 s, 1 substep) and at the benchmark's
    (1/60 s x 4 substeps).  The GPU reproduces the reference's trajectories
    bit for bit, so its errors are the reference algorithm's own: rolling is
    within 1 % of 5/7 g sin th; sliding is 5.1-5.3 % above g (sin th - mu cos th)
    at a 1/240 s substep (the XPBD friction's first-order discretisation
    error, identical in the reference), inside the reference's 10 % check."""
    g, ref = U.gpu(), U.oracle()
    for dt, sub in ((1.0 / 240.0, 1), (1.0 / 60.0, 4)):
        slide = checks52.sliding_acceleration_error(g, dt, sub)
        roll = checks52.rolling_acceleration_error(g, dt, sub)
        assert slide == checks52.sliding_acceleration_error(ref, dt, sub)
        assert roll == checks52.rolling_acceleration_error(ref, dt, sub)
        print("dt %.5f x %d substeps: sliding error %+.4f, rolling error %+.4f" % (dt, sub, slide, roll))
        assert abs(roll) < 0.01, roll
        assert abs(slide) < 0.1, slide


def test_reference_check_program_on_the_oracle():
    """The reference's own test program (test/test_main.cpp) linked against
    the oracle library: validates the oracle build."""
    import os
    import subprocess
    exe = os.path.join(U.ORACLE_DIR, "ref_checks.bin")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/ref_checks.bin not built (make -C oracle)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:]
    assert "52 checks, 0 failures" in r.stdout, r.stdout[-2000:]


@pytest.mark.gpu
def test_reference_check_program_on_the_gpu():
    """The reference's own test program, compiled unchanged against
    include/melon3d.h and linked with the GPU library: all 52 checks pass on
    the B200."""
    import os
    import subprocess
    exe = os.path.join(U.ORACLE_DIR, "ref_checks_gpu.bin")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/ref_checks_gpu.bin not built (make -C oracle gpu_checks)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout[-400:])
    assert r.returncode == 0, r.stdout[-2000:]
    assert "52 checks, 0 failures" in r.stdout, r.stdout[-2000:]
