"""LD loads and TL / NT two-ports on the device (loads.rs:103-222,
tl.rs:47-183, network.rs:55-142, applied as in solve_session.rs:1285-1309):
every load type's series impedance added to Z's diagonal, then the TL and
NT Z-parameter stamps, at each frequency before the Hallen solve.

Plain FP64 form vs the CPU oracle: the stamped diagonal bit for bit (the
host builds the same load values with the same num-complex operations),
pivots bit-exact, Zin and currents within 1e-9.  Mixed form: Zin within
1e-6 of the plain form.  The corpus's LD decks are covered with their
golden values by test_gpu_parity.py.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

# every load type, loads summing on one segment, a tag-0 card, a wire
# conductivity card (series below |gamma a| = 15, asymptotic above), an
# unsupported type and a sigma <= 0 card (both ignored)
WIRES = [(1, 31, (0, 0, 1.0), (0, 0, 9.0), 0.002), (2, 21, (1.5, 0, 1.2), (1.5, 0, 7.0), 0.001),
         (3, 11, (-2.0, 0, 3.0), (-2.0, 1.5, 5.0), 0.0015)]
SOURCES = [(1, 16, 1.0)]
LOADS = [(0, 1, 20, 20, 5.0, 2e-7, 3e-10), (1, 2, 10, 12, 300.0, 1e-6, 20e-12), (2, 3, 0, 0, 1.0, 1e-8, 0.0),
         (3, 1, 5, 0, 2.0, 0.0, 5e-10), (4, 1, 16, 16, 25.0, -12.0, 0.0), (5, 0, 0, 0, 3.5e7, 0.0, 0.0),
         (9, 1, 1, 1, 1.0, 1.0, 1.0), (5, 2, 1, 3, 0.0, 0.0, 0.0)]
FREQS = [3.0e6, 14.2e6, 29.7e6]


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _ant(acc, ground, loads=LOADS, freqs=FREQS, separate=False, sources=SOURCES):
    return acc.Antenna(acc.wires_array(WIRES), acc.sources_array(sources), freqs, ground, None,
                       separate_sources=separate, loads=None if loads is None else acc.loads_array(loads))


def test_stamped_diagonal_is_the_oracle_load_bit_for_bit(acc):
    segs = O.build_geometry(O.wires_array(WIRES))
    for ground in (0, 1):
        plain = acc.HallenBatch([_ant(acc, ground, loads=None)])
        plain.solve()
        loaded = acc.HallenBatch([_ant(acc, ground)])
        loaded.solve()
        for u, f in enumerate(FREQS):
            z0, zl = plain.read_z(u), loaded.read_z(u)
            lv, ign = O.build_loads(segs, f, O.loads_array(LOADS))
            assert ign == 4  # the unsupported card once, the sigma <= 0 card per segment
            d0 = np.ascontiguousarray(np.diag(z0))
            want = np.empty_like(d0)  # one separately rounded add per part
            want.real = d0.real + lv.real
            want.imag = d0.imag + lv.imag
            got = np.ascontiguousarray(np.diag(zl))
            assert np.array_equal(got.view(np.uint64), want.view(np.uint64))
            off = ~np.eye(len(segs), dtype=bool)
            assert np.array_equal(zl[off].view(np.uint64), z0[off].view(np.uint64))
        plain.close()
        loaded.close()


@pytest.mark.parametrize("ground", [0, 1])
def test_plain_matches_oracle_with_loads(acc, ground):
    b = acc.HallenBatch([_ant(acc, ground)])
    res = b.solve()
    for u, f in enumerate(FREQS):
        p = O.Problem(O.wires_array(WIRES), O.sources_array(SOURCES), f, ground=ground,
                      loads=O.loads_array(LOADS))
        O.solve_problem(p)
        assert p.status == 0 and res.status[u] == 0
        zg, zo = complex(*res.feeds[u][0, 5:7]), p.zin[0]
        assert abs(zg - zo) <= 1e-9 * abs(zo), (f, zg, zo)
        peak = np.abs(p.currents).max()
        assert np.abs(res.currents[u] - p.currents).max() <= 1e-9 * peak
        _, piv = b.read_unit(u)
        assert np.array_equal(piv, p.pivots[: len(piv)])
        # the loads change the answer
        q = O.Problem(O.wires_array(WIRES), O.sources_array(SOURCES), f, ground=ground)
        O.solve_problem(q)
        assert abs(q.zin[0] - zo) > 1e-3 * abs(zo)
    b.close()


def test_mixed_within_gate_with_loads(acc):
    ants = [_ant(acc, g) for g in (0, 1)]
    plain = acc.HallenBatch(ants, precision=acc.PRECISION_FP64).solve()
    b = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    mixed = b.solve()
    assert np.all(mixed.status == 0)
    for fm, fp in zip(mixed.feeds, plain.feeds):
        zm, zp = complex(*fm[0, 5:7]), complex(*fp[0, 5:7])
        assert abs(zm - zp) <= 1e-6 * abs(zp)
    b.close()


def test_loads_with_separate_sources_and_a_path_deck(acc):
    """Loads reuse one factorisation across right-hand sides, and apply to
    the conductor-path form (a start-to-start split dipole)."""
    srcs = [(1, 16, 1.0), (2, 5, 0.5j)]
    b = acc.HallenBatch([_ant(acc, 0, sources=srcs, separate=True, freqs=[14.2e6])])
    res = b.solve()
    for k, src in enumerate(srcs):
        p = O.Problem(O.wires_array(WIRES), O.sources_array([src]), 14.2e6, loads=O.loads_array(LOADS))
        O.solve_problem(p)
        assert abs(complex(*res.feeds[k][0, 5:7]) - p.zin[0]) <= 1e-9 * abs(p.zin[0])
    b.close()
    split = [(1, 26, (0, 0, 0), (0, 0, 5.282), 0.001), (2, 26, (0, 0, 0), (0, 0, -5.282), 0.001)]
    ld = [(2, 1, 1, 1, 20.0, 5e-7, 0.0), (5, 0, 0, 0, 5.8e7, 0.0, 0.0)]
    ant = acc.Antenna(acc.wires_array(split), acc.sources_array([(1, 1, 1.0)]), [14.2e6], 0, None,
                      loads=acc.loads_array(ld))
    res = acc.HallenBatch([ant]).solve()
    p = O.Problem(O.wires_array(split), O.sources_array([(1, 1, 1.0)]), 14.2e6, loads=O.loads_array(ld))
    O.solve_problem(p)
    assert abs(complex(*res.feeds[0][0, 5:7]) - p.zin[0]) <= 1e-9 * abs(p.zin[0])


# a lossless line (velocity factor 0.66) from wire 1 to wire 2's centre,
# a lossy line (2 dB), a line sharing the first one's end on wire 2 (a
# loaded segment), two ignored cards (coincident ends, z0 <= 0), and an NT
# two-port; stamps on one entry add in card order
TLS = [(1, 8, 2, 0, 1, 0, 75.0, 3.1, 0.66), (1, 24, 3, 6, 3, 1, 300.0, 7.5, 2.0), (2, 11, 3, 2, 0, 0, 450.0, 1.2, 1.0),
       (1, 5, 1, 5, 1, 0, 50.0, 1.0, 1.0), (1, 3, 2, 3, 1, 0, -50.0, 1.0, 1.0)]
NTS = [(1, 20, 2, 11, 0.002, -0.01, 0.0, 0.004, 0.001, -0.012)]


def _net_ant(acc, ground, freqs=FREQS):
    return acc.Antenna(acc.wires_array(WIRES), acc.sources_array(SOURCES), freqs, ground, None,
                       loads=acc.loads_array(LOADS), tls=acc.tls_array(TLS), nts=acc.nts_array(NTS))


def _oracle_net(f, ground):
    p = O.Problem(O.wires_array(WIRES), O.sources_array(SOURCES), f, ground=ground, loads=O.loads_array(LOADS),
                  tls=O.tls_array(TLS), nts=O.nts_array(NTS))
    return O.solve_problem(p)


def test_network_stamps_are_the_oracle_stamps_bit_for_bit(acc):
    segs = O.build_geometry(O.wires_array(WIRES))
    plain = acc.HallenBatch([_ant(acc, 0, loads=None)])
    plain.solve()
    stamped = acc.HallenBatch([_net_ant(acc, 0)])
    stamped.solve()
    for u, f in enumerate(FREQS):
        z = plain.read_z(u).copy()
        lv, _ = O.build_loads(segs, f, O.loads_array(LOADS))
        seq = [(i, i, lv[i]) for i in range(len(segs)) if lv[i] != 0]
        seq += O.tl_stamps(segs, f, O.tls_array(TLS)) + O.nt_stamps(segs, O.nts_array(NTS))
        assert len(O.tl_stamps(segs, f, O.tls_array(TLS))) == 12  # the two ignored cards stamp nothing
        for r, c, d in seq:  # separately rounded adds, in the reference's order
            v = z[r, c]
            z[r, c] = complex(v.real + d.real, v.imag + d.imag)
        got = stamped.read_z(u)
        assert np.array_equal(np.ascontiguousarray(got).view(np.uint64), z.view(np.uint64))
    plain.close()
    stamped.close()


@pytest.mark.parametrize("ground", [0, 1])
def test_plain_matches_oracle_with_networks(acc, ground):
    b = acc.HallenBatch([_net_ant(acc, ground)])
    res = b.solve()
    for u, f in enumerate(FREQS):
        p = _oracle_net(f, ground)
        assert p.status == 0 and res.status[u] == 0
        zg, zo = complex(*res.feeds[u][0, 5:7]), p.zin[0]
        assert abs(zg - zo) <= 1e-9 * abs(zo), (f, zg, zo)
        assert np.abs(res.currents[u] - p.currents).max() <= 1e-9 * np.abs(p.currents).max()
        _, piv = b.read_unit(u)
        assert np.array_equal(piv, p.pivots[: len(piv)])
    b.close()


def test_mixed_within_gate_with_networks(acc):
    ants = [_net_ant(acc, g) for g in (0, 1)]
    plain = acc.HallenBatch(ants, precision=acc.PRECISION_FP64).solve()
    b = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    mixed = b.solve()
    assert np.all(mixed.status == 0)
    for fm, fp in zip(mixed.feeds, plain.feeds):
        zm, zp = complex(*fm[0, 5:7]), complex(*fp[0, 5:7])
        assert abs(zm - zp) <= 1e-6 * abs(zp)
    b.close()
