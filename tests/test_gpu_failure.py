"""Failure detection on the B200 without a GPU fault: a kernel wait that can
never complete gives up after its limit, the kernel reports it, and the
device stays usable for the next step."""
from __future__ import annotations

import ctypes as C

import pytest

from simpletcsolver_b200 import abi, ic
from simpletcsolver_b200.solver import Solver

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_the_device_stays_usable(lib, tmp_path):
    sec = C.c_double(0.)
    assert lib.tcgpu_selftest_wait(C.byref(sec)) == 0, abi.last_error(lib)
    # the limit is about two seconds of SM clock
    assert 0.3 < sec.value < 30.0, sec.value
    case = ic.taylor_couette(16, 32, 16, 3400.0)
    s = Solver.from_ic(ic.write_ic(case, str(tmp_path / "ic")), case=case, lib=lib)
    try:
        assert s.integrate() > 0.0
        assert s.diagnostics()["divmax"] < 1e-12
    finally:
        s.release()
