"""The mixed form's fill evaluates the phase of its Gauss-Legendre samples,
e^{-jkR}, with its own sin(pi x), cos(pi x) (quadrant reduction and Taylor
series, fnec_mixed.cu fill_sincospi; the same source runs on the host
through a test hook).  Checked here against 50-digit mpmath values: the
error stays within a few units in the last place of 1 over the fill's
whole argument range, including the quadrant boundaries and the rounding
ties of the reduction."""
import numpy as np
import pytest

mpmath = pytest.importorskip("mpmath")


def _ref(x):
    mpmath.mp.dps = 50
    s = np.array([float(mpmath.sinpi(mpmath.mpf(v))) for v in x])
    c = np.array([float(mpmath.cospi(mpmath.mpf(v))) for v in x])
    return s, c


def test_fill_sincospi_matches_mpmath():
    import nec_accel as acc

    rng = np.random.default_rng(7)
    x = np.concatenate([
        rng.uniform(0.0, 1.0, 3000),
        rng.uniform(0.0, 64.0, 3000),
        rng.uniform(0.0, 4096.0, 1000),
        np.arange(0, 400) * 0.25,                       # quadrant boundaries (and f = +-1/4 ties)
        np.arange(0, 400) * 0.25 + 2.0 ** -40,
        np.nextafter(np.arange(1, 400) * 0.25, 0.0),
        [0.0, 1e-300, 5e-324, 1e-12, 0.5, 1.0, 1.5, 2.0, 2.0 ** 30 + 0.375],
    ])
    s, c = acc.test_fill_sincospi(x)
    rs, rc = _ref(x)
    assert np.max(np.abs(s - rs)) <= 4.5e-16
    assert np.max(np.abs(c - rc)) <= 4.5e-16
    # the pair stays on the unit circle to rounding
    assert np.max(np.abs(s * s + c * c - 1.0)) <= 1e-15


def test_fill_sincospi_refuses_out_of_range():
    import nec_accel as acc

    for bad in ([-1.0], [2.0 ** 50], [np.nan], [np.inf]):
        with pytest.raises(acc.AccelError):
            acc.test_fill_sincospi(np.array(bad))


@pytest.mark.gpu
def test_fill_rsqrt_matches_mpmath():
    """The fill's 1/sqrt(R^2) on the device (a single-precision guess and
    two Newton steps in FP64): within 4e-16 relative of 50-digit mpmath over
    the fill's range of R^2 and beyond."""
    import nec_accel as acc

    rng = np.random.default_rng(11)
    x = np.concatenate([np.exp(rng.uniform(np.log(1e-12), np.log(1e6), 4000)),
                        [1e-12, 2.5e-7, 1.0, 2.0, 4.0, 0.25, 1e4, 1e6]])
    y = acc.test_fill_rsqrt(x)
    mpmath.mp.dps = 50
    ref = np.array([float(1 / mpmath.sqrt(mpmath.mpf(v))) for v in x])
    assert np.max(np.abs(y - ref) / ref) <= 4e-16
    with pytest.raises(acc.AccelError):
        acc.test_fill_rsqrt(np.array([0.0]))
