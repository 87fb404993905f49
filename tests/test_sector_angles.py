"""Plane-sector angles: the engine's sector arithmetic against the host libm.

The reference takes a sample's plane sector from the host libm's atan2
(`(-d.x).atan2(d.y).rem_euclid(TAU)`, crates/estimation/src/search.rs:428-434).
The kernels take CUDA's atan2 and, within a few ulps of a sector boundary,
a correctly rounded double-double atan2 (boitata_b200/csrc/btk_turn.cuh).
Here the host build of that header is compared with the host libm (Python's
math.atan2 calls it) on random offsets and on offsets placed within a few
ulps of every boundary of 2 .. 360 sectors; disagreements are settled by a
60-digit atan2 from Python's decimal module. The host libm (glibc 2.39) is
not correctly rounded for about 1 input in 1,000, so at a boundary the
reference's sector depends on the platform it runs on; the engine takes
the correctly rounded value there.
"""

import ctypes
import math
import os
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def turn(tmp_path_factory):
    d = tmp_path_factory.mktemp("turn")
    src = d / "turn.cpp"
    src.write_text('#include "btk_turn.cuh"\n'
                   'extern "C" double t_atan2(double y, double x) { return btk::turn::atan2_rn(y, x); }\n'
                   'extern "C" int t_sector(double dx, double dy, int n) '
                   '{ return btk::turn::plane_sector(dx, dy, n); }\n')
    so = d / "turn.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-I",
                    os.path.join(ROOT, "boitata_b200", "csrc"), str(src), "-o", str(so)], check=True)
    lib = ctypes.CDLL(str(so))
    lib.t_atan2.restype, lib.t_atan2.argtypes = ctypes.c_double, [ctypes.c_double, ctypes.c_double]
    lib.t_sector.restype, lib.t_sector.argtypes = ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int]
    return lib


def atan2_60(y, x):
    """atan2 of two doubles to 60 digits (decimal arithmetic; atan by argument halving and its series)."""
    getcontext().prec = 70
    Y, X = Decimal(y), Decimal(x)
    ay, ax = abs(Y), abs(X)
    swap = ay > ax
    t = (ax / ay) if swap else (ay / ax)
    for _ in range(4):
        t = t / (1 + (1 + t * t).sqrt())
    s, term, k, t2 = Decimal(0), t, 0, t * t
    while abs(term) > Decimal(10) ** -68:
        s += term / (2 * k + 1) * (1 if k % 2 == 0 else -1)
        term *= t2
        k += 1
    a = 16 * s
    pi = Decimal("3.14159265358979323846264338327950288419716939937510582097494459230781640628620899863")
    if swap:
        a = pi / 2 - a
    if x < 0:
        a = pi - a
    return -a if y < 0 else a


def rounds_to(d60, v):
    """Whether the double v is the double nearest to d60."""
    lo, hi = np.nextafter(v, -np.inf), np.nextafter(v, np.inf)
    return abs(Decimal(v) - d60) <= min(abs(Decimal(lo) - d60), abs(Decimal(hi) - d60))


def boundary_offsets(n, rng, per=4):
    """Offsets (dx, dy) whose turn lies within a few ulps of each boundary of n sectors."""
    out = []
    for k in range(n):
        th = 2 * math.pi * k / n
        for _ in range(per):
            r = rng.uniform(0.5, 300.0)
            x, y = -r * math.sin(th), r * math.cos(th)
            x = float(np.nextafter(x, np.inf if rng.random() < 0.5 else -np.inf)) if x != 0 else x
            for _ in range(int(rng.integers(0, 4))):
                y = float(np.nextafter(y, np.inf if rng.random() < 0.5 else -np.inf))
            out.append((x, y))
    return out


def libm_misrounds(y, x):
    """Whether the host libm's atan2(y, x) is not the double nearest the exact value."""
    return not rounds_to(atan2_60(y, x), math.atan2(y, x))


def test_double_double_atan2_is_correctly_rounded(turn):
    """Where the header's atan2 and the host libm's differ, the header's is the correctly rounded one. The
    host libm (glibc) is not correctly rounded for about 1 input in 1,000."""
    rng = np.random.default_rng(7)
    ys = np.concatenate([rng.normal(size=20000) * 10.0 ** rng.uniform(-3, 3, 20000), rng.uniform(-1, 1, 5000)])
    xs = np.concatenate([rng.normal(size=20000) * 10.0 ** rng.uniform(-3, 3, 20000), rng.uniform(-1, 1, 5000)])
    bad = []
    for y, x in zip(ys.tolist(), xs.tolist()):
        if x == 0.0 or y == 0.0:
            continue
        got, want = turn.t_atan2(y, x), math.atan2(y, x)
        if got != want:
            bad.append((y, x, got, want))
    for y, x, got, want in bad:
        exact = atan2_60(y, x)
        assert rounds_to(exact, got) and not rounds_to(exact, want), (y, x, got, want)
    assert len(bad) <= 0.005 * len(ys)


@pytest.mark.parametrize("n", [2, 3, 4, 6, 8, 12, 36, 360])
def test_plane_sectors_near_every_boundary_are_the_references(turn, n):
    """The sector of offsets within a few ulps of every boundary is the reference's formula over the host
    libm, except where that libm's atan2 is not correctly rounded: there it is the formula over the
    correctly rounded atan2."""
    rng = np.random.default_rng(n)
    tau = 2 * math.pi

    def sector(at):
        t = at % tau  # Python's float % with a positive divisor is rem_euclid
        return min(int(t / tau * n), n - 1) if t / tau * n > 0 else 0

    for dx, dy in boundary_offsets(n, rng):
        got = turn.t_sector(dx, dy, n)
        if got != sector(math.atan2(-dx, dy)):
            assert libm_misrounds(-dx, dy), (dx, dy, n)
            assert got == sector(turn.t_atan2(-dx, dy))
