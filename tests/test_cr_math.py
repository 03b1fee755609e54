"""The correctly rounded sin/cos/ln/hypot of fnec_math.cuh (built for the
host with g++) against 256-bit mpmath, and their agreement with glibc (the
libm the reference's Rust f64 methods call)."""
import ctypes
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "fnec-rust_b200", "csrc")


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    out = tmp_path_factory.mktemp("probe") / "probe.so"
    subprocess.run(["g++", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-I", CSRC,
                    os.path.join(CSRC, "host_math_probe.cpp"), "-o", str(out)], check=True)
    L = ctypes.CDLL(str(out))
    P = ctypes.c_void_p
    L.probe_sincos.argtypes = [P, P, P, ctypes.c_long]
    L.probe_log.argtypes = [P, P, ctypes.c_long]
    L.probe_hypot.argtypes = [P, P, P, ctypes.c_long]
    return L


def test_sincos_correctly_rounded(probe):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 256
    rng = np.random.default_rng(7)
    x = np.concatenate([rng.uniform(-60, 60, 4000), rng.uniform(-1, 1, 1000) * 10.0 ** rng.uniform(-9, 0, 1000),
                        [np.pi / 2, np.pi, 1e-300, -0.0, 7e5, -9.9e5]])
    s = np.zeros_like(x)
    c = np.zeros_like(x)
    probe.probe_sincos(x.ctypes.data, s.ctypes.data, c.ctypes.data, len(x))
    bad = [v for i, v in enumerate(x) if float(mpmath.sin(mpmath.mpf(v))) != s[i]
           or float(mpmath.cos(mpmath.mpf(v))) != c[i]]
    assert not bad, bad[:5]
    # glibc agrees except where glibc itself is not correctly rounded
    agree = np.mean([math.sin(v) == s[i] and math.cos(v) == c[i] for i, v in enumerate(x)])
    assert agree > 0.99


def test_log_correctly_rounded(probe):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 256
    rng = np.random.default_rng(8)
    y = np.concatenate([rng.uniform(1, 1e5, 4000), 10.0 ** rng.uniform(-300, 300, 1000), [1.0, 2.0, 0.5]])
    o = np.zeros_like(y)
    probe.probe_log(y.ctypes.data, o.ctypes.data, len(y))
    bad = [v for i, v in enumerate(y) if float(mpmath.log(mpmath.mpf(v))) != o[i]]
    assert not bad, bad[:5]


def test_hypot_matches_glibc(probe):
    rng = np.random.default_rng(9)
    a = rng.uniform(-1e3, 1e3, 20000) * 10.0 ** rng.uniform(-8, 3, 20000)
    b = rng.uniform(-1e3, 1e3, 20000) * 10.0 ** rng.uniform(-8, 3, 20000)
    a = np.concatenate([a, [3.0, 0.0, 5e-200, 1e300, 1e-310]])
    b = np.concatenate([b, [4.0, 2.0, 7e-200, 1e300, 3e-310]])
    o = np.zeros_like(a)
    probe.probe_hypot(a.ctypes.data, b.ctypes.data, o.ctypes.data, len(a))
    bad = [(a[i], b[i]) for i in range(len(a)) if math.hypot(a[i], b[i]) != o[i]]
    assert not bad, bad[:5]
