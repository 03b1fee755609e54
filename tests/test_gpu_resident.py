"""Resident systems: new right-hand sides on a factorisation kept on the device.

The reference's accelerator keeps no device state between calls; the
north star's serving loop keeps Z and its factor on the device for extra
right-hand sides and pattern requests.  After a batch has run,
fnec_batch_set_sources + fnec_batch_resolve solve new voltage sources on
the stored factorisations (no fill, Gram or factor).  The plain form's
results must equal, bit for bit, a fresh batch planned with those sources;
the mixed form's must meet the 1e-6 gate against the plain form.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

WIRES = [(1, 31, (0.0, 0.0, 1.0), (0.0, 0.0, 11.0), 1e-3), (2, 25, (2.5, 0.0, 1.5), (2.5, 0.0, 10.0), 1.5e-3),
         (3, 21, (0.0, 0.0, 11.0), (3.0, 0.0, 13.0), 1e-3)]
FREQS = [13.5e6, 14.2e6, 21.1e6]
RP = (19, 3, 0.0, 0.0, 5.0, 60.0)


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _ant(acc, sources, separate, ground=1):
    return acc.Antenna(acc.wires_array(WIRES), acc.sources_array(sources), FREQS, ground, RP,
                       separate_sources=separate)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("separate", [False, True])
def test_plain_resolve_is_bit_identical_to_a_fresh_batch(acc, separate):
    first = [(1, 16, 1.0), (2, 13, 0.5j)]
    later = [(1, 4, 0.7 - 0.2j), (2, 20, 1.0)] if separate else [(1, 4, 0.7 - 0.2j), (2, 20, 1.0)]
    bt = acc.HallenBatch([_ant(acc, first, separate), _ant(acc, [(3, 11, 1.0)], False, ground=0)])
    r0 = bt.solve()
    bt.set_sources(0, later)
    r1 = bt.resolve()
    fresh = acc.HallenBatch([_ant(acc, later, separate), _ant(acc, [(3, 11, 1.0)], False, ground=0)])
    rf = fresh.solve()
    assert np.array_equal(r1.status, rf.status) and np.all(rf.status == 0)
    for u in range(len(rf.currents)):
        assert np.array_equal(_bits(r1.currents[u]), _bits(rf.currents[u])), u
        assert np.array_equal(_bits(r1.feeds[u]), _bits(rf.feeds[u])), u
        g1, gf = r1.pattern[u], rf.pattern[u]
        assert np.array_equal(_bits(g1[:, :4]), _bits(gf[:, :4])), u
    # the first sources again: the first run's results, bit for bit
    bt.set_sources(0, first)
    r2 = bt.resolve()
    for u in range(len(r0.currents)):
        assert np.array_equal(_bits(r2.currents[u]), _bits(r0.currents[u])), u
    bt.close()
    fresh.close()


def test_mixed_resolve_meets_the_gate(acc):
    first = [(1, 16, 1.0), (2, 13, 0.5j)]
    later = [(1, 27, 2.0), (2, 5, -1.0)]
    mixed = acc.HallenBatch([_ant(acc, first, True)], precision=acc.PRECISION_MIXED)
    mixed.solve()
    mixed.set_sources(0, later)
    rm = mixed.resolve()
    plain = acc.HallenBatch([_ant(acc, later, True)])
    rp = plain.solve()
    it, _ = mixed.refinement_stats()
    assert np.all(it > 0)
    for u in range(len(rp.currents)):
        zm = complex(*rm.feeds[u][0, 5:7])
        zp = complex(*rp.feeds[u][0, 5:7])
        assert abs(zm - zp) <= 1e-6 * abs(zp)
        assert np.linalg.norm(rm.currents[u] - rp.currents[u]) <= 1e-7 * np.linalg.norm(rp.currents[u])
    mixed.close()
    plain.close()


def test_resolve_refusals(acc):
    bt = acc.HallenBatch([_ant(acc, [(1, 16, 1.0), (2, 13, 1.0)], True)])
    with pytest.raises(acc.AccelError) as ei:  # no factorisation yet
        bt.resolve()
    assert ei.value.code == acc.ERR_BAD_ARG
    bt.solve()
    with pytest.raises(acc.AccelError) as ei:  # three right-hand sides where two were planned
        bt.set_sources(0, [(1, 16, 1.0), (2, 13, 1.0), (3, 2, 1.0)])
    assert ei.value.code == acc.ERR_BAD_ARG
    with pytest.raises(acc.AccelError) as ei:
        bt.set_sources(0, [(1, 99, 1.0), (2, 13, 1.0)])
    assert ei.value.code == acc.ERR_SEGMENT_NOT_FOUND
    with pytest.raises(acc.AccelError):
        bt.set_sources(1, [(1, 1, 1.0)])
    bt.close()
