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
