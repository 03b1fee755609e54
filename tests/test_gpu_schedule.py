"""Schedules, CUDA-graph replay and the autotuner (fnec_batch_*schedule*,
fnec_batch_graph_state, fnec_batch_tune, fnec_tune_cache_*).

The plain FP64 form must give the same bits under every schedule, eager or
replayed from a captured graph: a schedule only changes which kernels run
which units and how they are launched, never a unit's arithmetic.  The
mixed form must stay within the 1e-6 feedpoint gate of the plain form
under every schedule (every one refines to the same tolerance).
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    return nec_accel


def _ants(acc, n, seed, with_rp=False):
    rp = (19, 13, 0.0, 0.0, 5.0, 30.0) if with_rp else None
    return [acc.Antenna(acc.wires_array(w), acc.sources_array(src), [f], g, rp)
            for w, src, g, f in bench.uneven_workload(n, seed=seed)]


def _bits(res):
    cur = np.concatenate([c.view(np.uint64).ravel() for c in res.currents])
    feeds = np.concatenate([f.view(np.uint64).ravel() for f in res.feeds])
    pat = np.concatenate([p.view(np.uint64).ravel() for p in res.pattern]) if res.pattern else np.zeros(0, np.uint64)
    return cur, feeds, pat, np.asarray(res.status)


def _run(b, times=1):
    for _ in range(times):
        b.upload()
        b.run()
    b.sync()
    return b.read()


def _zin(res):
    return np.array([complex(*f[0, 5:7]) for f in res.feeds])


@pytest.fixture(scope="module")
def plain_ants(acc):
    ants = _ants(acc, 40, seed=31, with_rp=True)
    return ants


def test_plain_bits_equal_under_every_schedule(acc, plain_ants):
    b = acc.HallenBatch(plain_ants, precision=acc.PRECISION_FP64)
    assert b.info.max_s > 400  # some panels are taller than one CTA's shared memory
    b.schedule = {"graph": 0}
    ref = _bits(_run(b))
    assert np.all(ref[3] == 0)
    for sched in ({"grid_panels": 0}, {"grid_panels": 1, "class_shift": 2}, {"class_shift": 1, "graph": 2},
                  {"graph": 1}, {"grid_panels": 0, "class_shift": 2, "graph": 2}):
        b.schedule = sched
        got = _bits(_run(b, times=3))
        for r, g in zip(ref, got):
            assert np.array_equal(r, g), sched
    b.close()


def test_graph_capture_and_replay(acc, plain_ants):
    b = acc.HallenBatch(plain_ants[:12], precision=acc.PRECISION_FP64)
    b.schedule = {"graph": 1}
    assert b.graph_state() == (acc.GRAPH_NONE, 0)
    eager = _bits(_run(b))  # first run: eager
    assert b.graph_state()[0] == acc.GRAPH_NONE
    launches = b.kernel_launches
    replay = _bits(_run(b, times=4))  # captured at the second run, replayed after
    state, nodes = b.graph_state()
    assert state == acc.GRAPH_READY and nodes == launches == b.kernel_launches
    for r, g in zip(eager, replay):
        assert np.array_equal(r, g)
    b.schedule = {"class_shift": 2}  # a launch-shape change drops the graph
    assert b.graph_state()[0] == acc.GRAPH_NONE
    # profiled runs are eager (events between phases) and leave the graph alone
    b.schedule = {"class_shift": 1, "graph": 2}
    _run(b)
    assert b.graph_state()[0] == acc.GRAPH_READY
    b.set_profiling(True)
    b.run()
    ph = b.phase_ms()
    assert all(v >= 0 for v in ph.values())
    b.set_profiling(False)
    assert b.graph_state()[0] == acc.GRAPH_READY
    b.close()


def test_schedule_rejects_out_of_range(acc, plain_ants):
    b = acc.HallenBatch(plain_ants[:2], precision=acc.PRECISION_FP64)
    for bad in ({"class_shift": 3}, {"gmres_cluster": 3}, {"graph": 5}, {"grid_panels": -1}, {"factor_streams": 3},
                {"unit_factor": 4}, {"unit_factor": -1}, {"block_inverse": 5}, {"tensor_trailing": -1}, {"tensor_trailing": 3},
                {"gmres_ctas_per_sm": 2}, {"factor_pivoting": 2}, {"factor_pivoting": -1}):
        with pytest.raises(acc.AccelError) as e:
            b.schedule = bad
        assert e.value.code == acc.ERR_BAD_ARG
    b.close()


@pytest.mark.parametrize("sched", [
    {"gram_tensor": 0}, {"gram_tensor": 1},
    {"gmres_cluster": 2}, {"gmres_cluster": 4}, {"gmres_cluster": 8},
    {"gmres_cluster": 8, "gram_tensor": 0, "class_shift": 2, "graph": 2},
    {"factor_streams": 4}, {"factor_streams": 2, "class_shift": 2, "graph": 2},
    {"unit_factor": 0}, {"unit_factor": 1, "factor_streams": 4, "graph": 2},
    {"unit_factor": 2}, {"unit_factor": 3, "factor_streams": 2},
    {"block_inverse": 0}, {"block_inverse": 1, "gmres_cluster": 4},
    {"tensor_trailing": 0}, {"tensor_trailing": 1, "factor_streams": 4, "unit_factor": 0, "factor_pivoting": 1},
    {"tensor_trailing": 2, "factor_pivoting": 1},
    {"tensor_trailing": 2, "factor_streams": 4, "unit_factor": 0, "factor_pivoting": 1},
    {"gmres_ctas_per_sm": 4}, {"gmres_ctas_per_sm": 4, "block_inverse": 0},
    {"factor_pivoting": 1}, {"factor_pivoting": 1, "unit_factor": 3, "factor_streams": 2},
    {"factor_pivoting": 0, "unit_factor": 0, "factor_streams": 4, "class_shift": 2},
    {"factor_pivoting": 0, "unit_factor": 3, "block_inverse": 0},
])
def test_mixed_within_gate_under_every_schedule(acc, sched):
    ants = _ants(acc, 20, seed=32)  # few solves: clusters up to 8 CTAs fit
    plain = acc.HallenBatch(ants, precision=acc.PRECISION_FP64)
    zp = _zin(_run(plain))
    plain.close()
    b = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    b.schedule = sched
    got = b.schedule
    for k, v in sched.items():
        assert got[k] == v, (k, got)
    res = _run(b, times=3)
    assert np.all(res.status == 0)
    zm = _zin(res)
    assert np.max(np.abs(zm - zp) / np.abs(zp)) <= 1e-6
    b.close()


def test_tuner_sets_and_caches_the_fastest(acc, tmp_path):
    acc.tune_cache_clear()
    ants = _ants(acc, 48, seed=33)
    b = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    rep = b.tune(reps=2)
    assert rep["candidates"] >= 3 and not rep["from_cache"]
    assert 0 < rep["best_ms"] <= rep["default_ms"]
    assert b.schedule == rep["best"]
    assert acc.tune_cache_size() == 1
    res = _run(b, times=2)
    assert np.all(res.status == 0)
    b.close()
    # a batch of the same shape starts from the cached schedule
    b2 = acc.HallenBatch(_ants(acc, 48, seed=34), precision=acc.PRECISION_MIXED)
    r2 = b2.tune(reps=0)
    if r2["key"] == rep["key"]:
        assert r2["from_cache"] and b2.schedule == rep["best"]
    b2.close()
    path = tmp_path / "tune.txt"
    acc.tune_cache_save(path)
    acc.tune_cache_clear()
    acc.tune_cache_load(path)
    assert acc.tune_cache_size() == 1
    b3 = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    assert b3.schedule == rep["best"]  # applied at creation
    b3.close()
    acc.tune_cache_clear()


@pytest.mark.parametrize("pivoting", [0, 1])
def test_mixed_factor_groups_give_identical_bits(acc, pivoting):
    """Grouping units onto concurrent streams, or factoring small units whole
    in one CTA, changes only which launches run beside which: every unit's
    factor (the same operations in the same order), and so every solve, is
    the same -- for the Hermitian factor and for GEPP."""
    ants = _ants(acc, 32, seed=35)
    b = acc.HallenBatch(ants, precision=acc.PRECISION_MIXED)
    # all trailing updates as FP32 SIMT tiles: the whole-unit kernel repeats
    # the per-step kernels' arithmetic
    b.schedule = {"factor_streams": 1, "unit_factor": 0, "tensor_trailing": 0, "graph": 0,
                  "factor_pivoting": pivoting}
    ref = _bits(_run(b))
    for sched in ({"factor_streams": 2}, {"factor_streams": 4}, {"factor_streams": 4, "graph": 2},
                  {"unit_factor": 1, "factor_streams": 1}, {"unit_factor": 1, "factor_streams": 4},
                  {"unit_factor": 3, "factor_streams": 2}):
        b.schedule = sched
        got = _bits(_run(b, times=2))
        for r, g in zip(ref, got):
            assert np.array_equal(r, g), sched
    if pivoting == 0:
        b.close()
        return
    # tensor-core trailing updates: the same units take them in every grouping
    b.schedule = {"factor_streams": 1, "unit_factor": 1, "tensor_trailing": 1, "graph": 0}
    ref = _bits(_run(b))
    for sched in ({"factor_streams": 2}, {"factor_streams": 4, "graph": 2}):
        b.schedule = sched
        got = _bits(_run(b, times=2))
        for r, g in zip(ref, got):
            assert np.array_equal(r, g), sched
    b.close()


@pytest.mark.parametrize("pivoting", [1, 0])
@pytest.mark.parametrize("cells", [9, 12, 16])
def test_tensor_core_trailing_keeps_the_refinement(acc, cells, pivoting):
    """The factor's trailing updates on tcgen05 (3xTF32) give a preconditioner
    as good as the FP32 SIMT one: the same answer within the gate and no more
    than one extra refinement iteration -- for GEPP and for the Hermitian
    factor (tiles on and below the diagonal only)."""
    wl, src, f = bench.mesh_workload(cells)
    ant = [acc.Antenna(acc.wires_array(wl), acc.sources_array(src), [f], acc.GROUND_PEC, None)]
    plain = acc.HallenBatch(ant, precision=acc.PRECISION_FP64)
    zp = _zin(_run(plain))[0]
    plain.close()
    out = {}
    for tt in (0, 1):
        b = acc.HallenBatch(ant, precision=acc.PRECISION_MIXED)
        assert b.info.max_s - 32 >= 192
        b.schedule = {"tensor_trailing": tt, "factor_pivoting": pivoting}
        res = _run(b)
        assert np.all(res.status == 0)
        it, rs = b.refinement_stats()
        out[tt] = (_zin(res)[0], int(it.max()))
        b.close()
    for tt, (zm, it) in out.items():
        assert abs(zm - zp) <= 1e-6 * abs(zp), tt
    assert out[1][1] <= out[0][1] + 1


def test_read_report_equals_the_full_read():
    """fnec_batch_read_report: the packed 4 pattern columns, currents, feeds
    and status are the full read's, bit for bit."""
    import nec_accel as acc

    nec = acc
    wires = [(1, 21, (0, 0, -2.5), (0, 0, 2.5), 0.001), (2, 15, (1.0, 0, -2.0), (1.0, 0, 2.0), 0.001)]
    ant = nec.Antenna(nec.wires_array(wires), nec.sources_array([(1, 11, 1.0)]), [14.2e6, 21.0e6], 0,
                      (10, 7, 0.0, 0.0, 20.0, 60.0))
    b = nec.HallenBatch([ant])
    b.run()
    b.sync()
    cur, feed, pat, st, _ = [x.copy() for x in b.read_raw()]
    cur4, feed4, pat4, st4 = [x.copy() for x in b.read_report()]
    assert np.array_equal(pat4.view(np.uint64), np.ascontiguousarray(pat[:, :4]).view(np.uint64))
    assert np.array_equal(cur4.view(np.uint64), cur.view(np.uint64))
    assert np.array_equal(feed4.view(np.uint64), feed.view(np.uint64)) and np.array_equal(st4, st)
    # the streamed run: the same columns, copied chunk by chunk behind the far field
    b._pat4[:] = 0.0
    b.run_report()
    cur5, feed5, pat5, st5 = [x.copy() for x in b.read_report(pattern=False)]
    assert np.array_equal(pat5.view(np.uint64), pat4.view(np.uint64))
    assert np.array_equal(cur5.view(np.uint64), cur.view(np.uint64)) and np.array_equal(st5, st)
    b.close()
