"""The traversal divides by direction components with div_recip (a
reciprocal per ray and two Markstein corrections) instead of a full IEEE
division per step. These tests check that method against IEEE division on
the host, so the oracle's plain divisions and the GPU's agree bit for bit."""
import ctypes
import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("division") / "division_check.so"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-shared", "-fPIC",
                    os.path.join(HERE, "division_check.c"), "-o", str(out), "-lm"], check=True)
    so = ctypes.CDLL(str(out))
    for name in ("check_random", "check_midpoints"):
        getattr(so, name).restype = ctypes.c_uint64
        getattr(so, name).argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)]
    so.check_binade.restype = ctypes.c_uint64
    so.check_binade.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]
    return so


def test_random_quotients_round_like_ieee_division(lib):
    bad = (ctypes.c_float * 2)()
    assert lib.check_random(20_000_000, 12345, bad) == 0, (bad[0], bad[1])


def test_quotients_near_rounding_midpoints_round_like_ieee_division(lib):
    bad = (ctypes.c_float * 2)()
    assert lib.check_midpoints(20_000_000, 777, bad) == 0, (bad[0], bad[1])


@pytest.mark.parametrize("a,lo", [(1.0, 0.5), (-15.999, 0.5), (0.0015, 2.0 ** -27), (7.25, 2.0 ** -12), (1000.5, 0.25)])
def test_every_divisor_of_a_binade_rounds_like_ieee_division(lib, a, lo):
    bad = (ctypes.c_float * 2)()
    assert lib.check_binade(a, lo, bad) == 0, (bad[0], bad[1])
