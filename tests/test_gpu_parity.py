"""Parity of the plain FP64 CUDA path with the CPU oracle (run on a B200).

Bars (from the task's parity contract):
  * segment indexing, junction connectivity, pivot order: bit-exact;
  * feedpoint Zin: |dZ|/|Z| <= 1e-9;
  * segment currents: max|dI| / max|I| <= 1e-9 (normwise; the free-end
    currents are ~1e-5 of the peak and carry the cancellation of the
    ill-conditioned normal equations, so an elementwise bar would measure
    the conditioning, not the port);
  * gains: |dG| <= 1e-6 dB wherever the oracle's gain is above the
    -999.99 clamp, and the clamp itself identical.
Given the oracle's own Z, the device Gram + elimination + back substitution
must reproduce the oracle's solution bit for bit.
"""
import numpy as np
import pytest

from _corpus import deck_arrays, deck_loads, deck_networks, golden_zins, load_cases
from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = load_cases()
ZIN_TOL = 1e-9
CUR_TOL = 1e-9
GAIN_TOL_DB = 1e-6


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _antenna(acc, deck, freqs=None, rp=None):
    wires, sources, _ = deck_arrays(deck)
    rp = rp if rp is not None else (tuple(deck["rp"]) if deck.get("rp") else None)
    ld = deck_loads(deck)
    tl, nt = deck_networks(deck)
    return acc.Antenna(wires.view(acc.WIRE_DTYPE), sources.view(acc.SOURCE_DTYPE),
                       freqs if freqs is not None else deck["freqs"], deck["ground"], rp,
                       loads=None if ld is None else ld.view(acc.LOAD_DTYPE),
                       tls=None if tl is None else tl.view(acc.TL_DTYPE),
                       nts=None if nt is None else nt.view(acc.NT_DTYPE))


def _check_unit(acc, batch, res, u, wires, sources, ground, freq, pts, loads=None, cur_tol=CUR_TOL, tls=None,
                nts=None, zin_tol=ZIN_TOL, bit_exact=False, solved=None):
    p = solved
    if p is None:
        p = O.Problem(wires, sources, freq, ground=ground, points=pts, loads=loads, tls=tls, nts=nts)
        O.solve_problem(p)
    assert p.status == 0
    assert res.status[u] == 0
    feeds = res.feeds[u]
    assert len(feeds) == len(p.zin)
    for row, zr in zip(feeds, p.zin):
        zg = complex(row[5], row[6])
        assert abs(zg - zr) <= zin_tol * abs(zr), (zg, zr)
    cur = res.currents[u]
    peak = np.abs(p.currents).max()
    if peak == 0.0:  # every segment is a constrained free end (a 1-segment wire)
        assert np.array_equal(cur, p.currents)
    else:
        assert np.abs(cur - p.currents).max() / peak <= cur_tol
    if bit_exact:
        # the fill's sin/cos/hypot are the platform libm's and its ln is the
        # host's, so the whole solve reproduces the oracle bit for bit
        assert np.array_equal(cur.view(np.uint64), p.currents.view(np.uint64)), \
            np.abs(cur - p.currents).max() / max(peak, 1e-300)
        zg = np.array([complex(r[5], r[6]) for r in feeds])
        assert np.array_equal(zg.view(np.uint64), np.asarray(p.zin, np.complex128).view(np.uint64))
    _, piv = batch.read_unit(u)
    # the oracle's pivot buffer has room for n + (GW cards) rows; the solve
    # uses n + (columns): merged wires, or conductor paths in the path form
    assert len(piv) == batch.units[u]["s"] <= len(p.pivots)
    assert np.array_equal(piv, p.pivots[: len(piv)])
    if pts is not None:
        g = res.pattern[u][:, :4]
        ref = p.pattern
        clamp = ref[:, 0] <= -999.0
        assert np.array_equal(g[clamp, 0], ref[clamp, 0])
        live = ~clamp
        assert np.abs(g[live, 0] - ref[live, 0]).max(initial=0) <= GAIN_TOL_DB
        for col in (1, 2):
            ok = ref[:, col] > -999.0
            assert np.abs(g[ok, col] - ref[ok, col]).max(initial=0) <= GAIN_TOL_DB
            assert np.array_equal(g[~ok, col], ref[~ok, col])
        assert np.abs(g[:, 3] - ref[:, 3]).max() <= 1e-9
    return p


@pytest.mark.parametrize("name", sorted(CASES))
def test_corpus_case_matches_oracle_and_golden(acc, name):
    case = CASES[name]
    deck = case["deck"]
    wires, sources, pts = deck_arrays(deck)
    batch = acc.HallenBatch([_antenna(acc, deck)])
    res = batch.solve()
    golden = golden_zins(case)
    for u, f in enumerate(deck["freqs"]):
        tl, nt = deck_networks(deck)
        _check_unit(acc, batch, res, u, wires, sources, deck["ground"], f, pts, loads=deck_loads(deck),
                    tls=tl, nts=nt, bit_exact=True)
        if f in golden:
            for row, want in zip(res.feeds[u], golden[f]):
                got = complex(row[5], row[6])
                tol = 2e-6 if len(repr(want.real).split(".")[-1]) >= 6 else 0.05
                assert abs(got.real - want.real) <= tol and abs(got.imag - want.imag) <= tol


def _oracle_stamped_z(segs, f, ground, deck):
    """The oracle's Z with the deck's LD loads on the diagonal, then its TL
    and NT stamps in card order (solve_session.rs:1285-1309), each stamp one
    separately rounded add per part."""
    z = O.assemble_z(segs, f, ground)
    ld = deck_loads(deck)
    if ld is not None:
        lv, _ = O.build_loads(segs, f, ld)
        for i in range(len(segs)):
            z[i, i] = complex(z[i, i].real + lv[i].real, z[i, i].imag + lv[i].imag)
    tl, nt = deck_networks(deck)
    for r, c, d in (O.tl_stamps(segs, f, tl) if tl is not None else []) + \
            (O.nt_stamps(segs, nt) if nt is not None else []):
        z[r, c] = complex(z[r, c].real + d.real, z[r, c].imag + d.imag)
    return z


@pytest.mark.parametrize("name", sorted(CASES))
def test_z_fill_bit_identical_to_oracle(acc, name):
    """matrix.rs fill (elem + green_k + image terms, matrix.rs:186-331,
    :397) and the LD/TL/NT stamps: with glibc's sin/cos restated on the
    device and the self term's ln taken from the host libm, every element of
    Z equals the oracle's bit for bit, in free space and over PEC ground."""
    deck = CASES[name]["deck"]
    wires, sources, _ = deck_arrays(deck)
    segs = O.build_geometry(wires)
    grounds = (0, 1) if name == "yagi-5elm-51seg" else (deck["ground"],)
    for ground in grounds:
        d = dict(deck, ground=ground, rp=None)
        batch = acc.HallenBatch([_antenna(acc, d)])
        batch.solve()
        for u, f in enumerate(deck["freqs"]):
            zg = batch.read_z(u)
            zr = _oracle_stamped_z(segs, f, ground, deck)
            assert np.array_equal(zg.view(np.uint64), zr.view(np.uint64)), \
                (f, np.mean(zg.view(np.uint64) == zr.view(np.uint64)), np.abs(zg - zr).max())
        batch.close()


def test_solve_is_bit_exact_given_the_oracle_z(acc):
    """Gram (linear.rs:765-785), GEPP (:1343-1370) and back substitution
    (:1372-1381) reproduce the oracle bit for bit on the same inputs."""
    for name in ("yagi-5elm-51seg", "dipole-ground-51seg", "multi-source", "dipole-loaded", "tl-two-dipoles-linked",
                 "tl-two-dipoles-linked-seg0-even52", "dipole-nt-tl-equiv-freesp-51seg"):
        deck = CASES[name]["deck"]
        wires, sources, _ = deck_arrays(deck)
        segs = O.build_geometry(wires)
        f = deck["freqs"][0]
        rhs, cosv = O.hallen_rhs(segs, f, sources)
        z = O.assemble_z(segs, f, deck["ground"])
        tl, nt = deck_networks(deck)  # the oracle's two-port stamps, in order
        for r, c, d in (O.tl_stamps(segs, f, tl) if tl is not None else []) + \
                (O.nt_stamps(segs, nt) if nt is not None else []):
            z[r, c] = complex(z[r, c].real + d.real, z[r, c].imag + d.imag)
        m = O.merge_collinear(segs)
        ja, jb, js = O.cli_junctions(segs, m)
        x0, p0 = O.solve_hallen(z, rhs, cosv, m, ja, jb, js)
        x1, p1 = acc.solve_hallen(z, rhs, cosv, m, list(zip(ja, jb, js)), return_pivots=True)
        assert np.array_equal(p0, p1)
        assert np.array_equal(x0.view(np.uint64), x1.view(np.uint64)), np.abs(x0 - x1).max()


def test_junction_geometry_bit_exact_solve_and_connectivity(acc):
    """T-junction (3 wire ends at one node) + a bend: pairwise junction rows
    (geometry.rs:274-339) and the constraint-row Gram terms."""
    wires = O.wires_array([(1, 7, (0, 0, 0.3), (0, 0, 2.0), 1e-3), (2, 5, (0, 0, 2.0), (1.5, 0, 2.0), 1e-3),
                           (3, 6, (1.5, 0, 2.0), (1.5, 0, 0.2), 1e-3), (4, 3, (0, 0, 2.0), (-1, 0, 2.5), 1e-3)])
    sources = O.sources_array([(1, 4, 1.0)])
    segs = O.build_geometry(wires)
    for ground in (0, 1):
        batch = acc.HallenBatch([acc.Antenna(wires.view(acc.WIRE_DTYPE), sources.view(acc.SOURCE_DTYPE),
                                             [30e6], ground, (19, 2, 0.0, 0.0, 10.0, 90.0))])
        res = batch.solve()
        _check_unit(acc, batch, res, 0, wires, sources, ground, 30e6, O.rp_card_points(19, 2, 0, 0, 10, 90))
        rhs, cosv = O.hallen_rhs(segs, 30e6, sources)
        z = O.assemble_z(segs, 30e6, ground)
        m = O.merge_collinear(segs)
        ja, jb, js = O.cli_junctions(segs, m)
        assert len(ja) == 4
        x0, p0 = O.solve_hallen(z, rhs, cosv, m, ja, jb, js)
        x1, p1 = acc.solve_hallen(z, rhs, cosv, m, list(zip(ja, jb, js)), return_pivots=True)
        assert np.array_equal(x0.view(np.uint64), x1.view(np.uint64))
        assert np.array_equal(p0, p1)


def five_wire_array(seed=11, nseg=51, f0=14.2e6):
    """The 5-element parallel-wire array of the sweep workload: lengths
    U(0.9, 1.1) * lambda/2, x gaps U(0.15, 0.25) * lambda, r = 1 mm."""
    rng = np.random.default_rng(seed)
    lam = 299792458.0 / f0
    x = 0.0
    wires = []
    for t in range(5):
        L = rng.uniform(0.9, 1.1) * lam / 2
        wires.append((t + 1, nseg, (x, 0.0, -L / 2), (x, 0.0, L / 2), 1e-3))
        x += rng.uniform(0.15, 0.25) * lam
    return O.wires_array(wires), O.sources_array([(2, (nseg + 1) // 2, 1.0)])


def test_sweep_batch_with_full_pattern_grid(acc):
    """Several frequencies of the 5-wire array in one batch with the
    91 x 361 RP grid: every unit matches the oracle."""
    wires, sources = five_wire_array()
    freqs = [13.0e6, 14.25e6, 15.5e6]
    rp = (91, 361, 0.0, 0.0, 1.0, 1.0)
    batch = acc.HallenBatch([acc.Antenna(wires.view(acc.WIRE_DTYPE), sources.view(acc.SOURCE_DTYPE), freqs,
                                         0, rp)])
    res = batch.solve()
    pts = O.rp_card_points(*rp)
    for u, f in enumerate(freqs):
        _check_unit(acc, batch, res, u, wires, sources, 0, f, pts)


def test_uneven_multi_antenna_batch(acc):
    """Antennas of different N, ground and source placement in one batch;
    each unit equals its solve alone."""
    rng = np.random.default_rng(5)
    ants = []
    refs = []
    for a in range(6):
        nw = int(rng.integers(1, 4))
        wl = []
        for t in range(nw):
            p0 = rng.uniform(-3, 3, 3)
            p0[2] = rng.uniform(0.5, 4)
            p1 = p0 + rng.uniform(-2, 2, 3)
            p1[2] = max(p1[2], 0.3)
            wl.append((t + 1, int(rng.integers(3, 21)) * 2 + 1, tuple(p0), tuple(p1), 10 ** rng.uniform(-3.3, -2.3)))
        w = O.wires_array(wl)
        s = O.sources_array([(1, (wl[0][1] + 1) // 2, 1.0)])
        ground = int(a % 2)
        f = float(10 ** rng.uniform(np.log10(3e6), np.log10(30e6)))
        ants.append(acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], ground,
                                (7, 5, 0.0, 0.0, 30.0, 72.0)))
        refs.append((w, s, ground, f))
    batch = acc.HallenBatch(ants)
    res = batch.solve()
    for u, (w, s, ground, f) in enumerate(refs):
        _check_unit(acc, batch, res, u, w, s, ground, f, O.rp_card_points(7, 5, 0, 0, 30, 72))


def test_single_segment_and_error_statuses(acc):
    w = O.wires_array([(1, 1, (0, 0, -0.5), (0, 0, 0.5), 1e-3)])
    s = O.sources_array([(1, 1, 1.0)])
    batch = acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [100e6])])
    res = batch.solve()
    _check_unit(acc, batch, res, 0, w, s, 0, 100e6, None)
    bad = O.sources_array([(1, 2, 1.0)])
    with pytest.raises(acc.AccelError) as ei:
        acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), bad.view(acc.SOURCE_DTYPE), [100e6])])
    assert ei.value.code == acc.ERR_SEGMENT_NOT_FOUND
    zero = O.wires_array([(1, 3, (0, 0, 1), (0, 0, 1), 1e-3)])
    with pytest.raises(acc.AccelError) as ei:
        acc.HallenBatch([acc.Antenna(zero.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [100e6])])
    assert ei.value.code == acc.ERR_BAD_ARG


def test_reference_entry_points(acc):
    """fill_zmatrix_wgpu / solve_hallen_gpu_resident / run_rp_farfield_batch
    equivalents against the oracle."""
    deck = CASES["dipole-ground-51seg"]["deck"]
    wires, sources, _ = deck_arrays(deck)
    segs = O.build_geometry(wires)
    f = deck["freqs"][0]
    zseg = acc.zsegments_from(segs)
    for ground in (0, 1):
        z = acc.fill_zmatrix(zseg, f, ground)
        zr = O.assemble_z(segs, f, ground)
        assert np.abs(z - zr).max() / np.abs(zr).max() < 1e-14
    rhs, cosv = O.hallen_rhs(segs, f, sources)
    m = O.merge_collinear(segs)
    x, piv = acc.solve_hallen_gpu_resident(zseg, rhs, cosv, m, [], f, ground=1, return_pivots=True)
    x0, p0 = O.solve_hallen(O.assemble_z(segs, f, 1), rhs, cosv, m, [], [], [])
    assert np.abs(x - x0).max() / np.abs(x0).max() <= CUR_TOL and np.array_equal(piv, p0)
    gseg = acc.gpu_segments_from(segs)
    pts = O.rp_card_points(10, 4, 0.0, 0.0, 10.0, 90.0)
    out, tot = acc.compute_radiation_pattern(gseg, x0[: len(segs)], f, pts, ground=1)
    ref, tot_ref = O.radiation_pattern(segs, x0[: len(segs)], f, pts, ground=1)
    assert abs(tot - tot_ref) / tot_ref < 1e-12
    live = ref[:, 0] > -999
    assert np.abs(out[live, 0] - ref[live, 0]).max() <= GAIN_TOL_DB
    # run_rp_farfield_batch_wgpu has no ground argument: free space, with
    # the caller's normalisation
    k = 2 * np.pi / (299792458.0 / f)
    ref_free, tot_free = O.radiation_pattern(segs, x0[: len(segs)], f, pts, ground=0)
    r = acc.run_rp_farfield_batch(gseg, x0[: len(segs)], k, tot_free, pts)
    live_f = ref_free[:, 0] > -999
    assert np.abs(r["gain_total_dbi"][live_f] - ref_free[live_f, 0]).max() <= GAIN_TOL_DB
    assert np.abs(r["axial_ratio"] - ref_free[:, 3]).max() <= 1e-9
    assert abs(acc.integrate_radiated_power(gseg, x0[: len(segs)], f, True) - tot_ref) / tot_ref < 1e-12
    mb = acc.microbench_zmatrix_dispatch(160, 5)
    assert mb.dispatch_median_us > 0
    assert acc.enumerate_compute_adapters()[0]["name"]
    assert acc.dispatch_frequency_point(acc.GPU_ONLY, f) == "RunOnGpu"


def test_uneven_random_antenna_batch_sample(acc):
    """64 antennas of the uneven 4096-antenna workload generator in one
    batch (N from tens to hundreds, free space and GN 1 mixed)."""
    import bench

    wl = bench.uneven_workload(64, seed=7)
    ants = [acc.Antenna(acc.wires_array(w), acc.sources_array(s), [f], g, None) for w, s, g, f in wl]
    batch = acc.HallenBatch(ants)
    res = batch.solve()
    for u in range(0, 64, 7):
        w, s, g, f = wl[u]
        _check_unit(acc, batch, res, u, O.wires_array(w), O.sources_array(s), g, f, None)


def test_extra_right_hand_sides_reuse_the_factor_bit_exactly(acc):
    """separate_sources: three source positions on one factorisation per
    frequency.  Solve r must be bit-identical to the single-source deck
    solved on its own (the reference re-runs the whole elimination for a
    new source; only the b column differs), and match the oracle."""
    wl = [(1, 21, (0, 0, 1.0), (0, 0, 6.0), 1e-3), (2, 15, (1.2, 0, 1.0), (1.2, 0, 5.0), 1e-3),
          (3, 9, (0, 0, 6.0), (1.2, 0, 6.5), 1e-3)]
    srcs = [(1, 11, 1.0), (2, 8, 0.5 - 0.25j), (3, 2, 1.0)]
    w = O.wires_array(wl)
    freqs = [20e6, 26e6]
    for ground in (0, 1):
        multi = acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), O.sources_array(srcs).view(acc.SOURCE_DTYPE),
                                             freqs, ground, (9, 3, 0.0, 0.0, 10.0, 60.0), separate_sources=True)])
        rm = multi.solve()
        assert len(rm.currents) == len(freqs) * len(srcs)
        for fi, f in enumerate(freqs):
            for r, src in enumerate(srcs):
                one = acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), O.sources_array([src]).view(acc.SOURCE_DTYPE),
                                                   [f], ground, (9, 3, 0.0, 0.0, 10.0, 60.0))])
                ro = one.solve()
                u = fi * len(srcs) + r
                xm, _ = multi.read_unit(u)
                xo, _ = one.read_unit(0)
                assert np.array_equal(xm.view(np.uint64), xo.view(np.uint64)), (fi, r)
                assert np.array_equal(rm.feeds[u], ro.feeds[0])
                assert np.array_equal(rm.pattern[u], ro.pattern[0])
                _check_unit(acc, one, ro, 0, w, O.sources_array([src]), ground, f,
                            O.rp_card_points(9, 3, 0, 0, 10, 60))


@pytest.mark.parametrize("cells", [3, 6])
def test_junctioned_mesh_over_ground(acc, cells):
    """The mesh workload at small size: every interior node joins four wire
    ends (6 pairwise junction rows each), GN 1 images, bit-exact solve given
    the oracle's Z, and end-to-end parity."""
    import bench

    wl, src, f = bench.mesh_workload(cells)
    w = O.wires_array(wl)
    s = O.sources_array(src)
    batch = acc.HallenBatch([acc.Antenna(w.view(acc.WIRE_DTYPE), s.view(acc.SOURCE_DTYPE), [f], 1,
                                         (10, 4, 0.0, 0.0, 10.0, 90.0))])
    res = batch.solve()
    _check_unit(acc, batch, res, 0, w, s, 1, f, O.rp_card_points(10, 4, 0, 0, 10, 90))
    segs = O.build_geometry(w)
    rhs, cosv = O.hallen_rhs(segs, f, s)
    z = O.assemble_z(segs, f, 1)
    m = O.merge_collinear(segs)
    ja, jb, js = O.cli_junctions(segs, m)
    x0, p0 = O.solve_hallen(z, rhs, cosv, m, ja, jb, js)
    x1, p1 = acc.solve_hallen(z, rhs, cosv, m, list(zip(ja, jb, js)), return_pivots=True)
    assert np.array_equal(p0, p1)
    assert np.array_equal(x0.view(np.uint64), x1.view(np.uint64))
