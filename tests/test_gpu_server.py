"""The serving loop (fnec_server_*): continuous batching over CUDA-stream
lanes with admission by HBM budget.

Each request is a random antenna deck with 1-4 source positions (separate
right-hand sides on one factorisation) and an optional 91 x 361 pattern.
Requests submitted together are batched and their batches overlap on the
device; every result must equal the result of solving that deck alone:
bit for bit in the plain FP64 form (its per-unit arithmetic does not depend
on what else is in the batch), and within the 1e-6 feedpoint gate in the
mixed form.
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    return nec_accel


def _antennas(acc, n, seed, n_cap=400):
    out = []
    for wires, srcs, ground, f, rp in bench.serve_requests(n, seed=seed, n_cap=n_cap):
        out.append(acc.Antenna(acc.wires_array(wires), acc.sources_array(srcs), [f], ground, rp,
                               separate_sources=True))
    return out


def _serve(acc, ants, precision, **kw):
    """Serve every deck at once; every other request gets its results copied
    into its own arrays, the rest read them in place before release.
    Returns per request (currents, feeds, pattern, status) copies, the
    latencies and the server statistics."""
    with acc.Server(precision, **kw) as srv:
        reqs = [srv.submit(a, copy_out=(i % 2 == 0)) for i, a in enumerate(ants)]
        out, lat = [], []
        for r in reqs:
            srv.wait(r)
            out.append(tuple(None if x is None else np.array(x, copy=True) for x in r.result()))
            lat.append(r.latency_ms)
            r.release()
        stats = srv.stats()
    return out, lat, stats


def _alone(acc, a, precision):
    b = acc.HallenBatch([a], precision=precision)
    res = b.solve()
    b.close()
    return res


def test_server_fp64_results_equal_solving_alone(acc):
    ants = _antennas(acc, 16, seed=21)
    outs, lat, stats = _serve(acc, ants, acc.PRECISION_FP64, lanes=2, max_batch=6)
    assert stats["completed"] == len(ants) and stats["failed"] == 0
    assert stats["batches"] >= 3  # 16 requests, at most 6 per batch
    for a, (cur, feeds, pat, status), ms in zip(ants, outs, lat):
        res = _alone(acc, a, acc.PRECISION_FP64)
        assert len(cur) == len(res.currents) == len(a.sources)
        assert np.array_equal(status, res.status)
        for k in range(len(cur)):
            assert np.array_equal(cur[k].view(np.uint64), res.currents[k].view(np.uint64))
        assert np.array_equal(feeds, np.concatenate(res.feeds))
        if pat is not None:
            for k in range(len(cur)):
                assert np.array_equal(pat[k], res.pattern[k])
        assert ms is not None and ms > 0.0


def test_server_mixed_results_within_gate(acc):
    ants = _antennas(acc, 12, seed=22)
    mixed, _, stats = _serve(acc, ants, acc.PRECISION_MIXED, lanes=3, max_batch=4)
    plain, _, _ = _serve(acc, ants, acc.PRECISION_FP64, lanes=1, max_batch=12)
    assert stats["completed"] == len(ants)
    for a, rm, rp in zip(ants, mixed, plain):
        alone = _alone(acc, a, acc.PRECISION_MIXED)
        n_solves = len(rm[0])
        rows = len(rm[1]) // n_solves
        for k in range(n_solves):
            zm = complex(*rm[1][k * rows, 5:7])
            zp = complex(*rp[1][k * rows, 5:7])
            za = complex(*alone.feeds[k][0, 5:7])
            assert abs(zm - zp) <= 1e-6 * abs(zp)
            assert abs(zm - za) <= 1e-6 * abs(za)


def test_server_admission_respects_budget(acc):
    ants = _antennas(acc, 10, seed=23)
    with acc.Server(acc.PRECISION_FP64, lanes=2, max_batch=8) as probe:
        need = [probe.shape(a).device_bytes for a in ants]
    budget = max(need)
    outs, _, stats = _serve(acc, ants, acc.PRECISION_FP64, lanes=2, max_batch=8, hbm_budget_bytes=budget)
    assert stats["completed"] == len(ants)
    assert stats["peak_in_flight_bytes"] <= budget
    assert all(np.all(o[3] == 0) for o in outs)


def test_server_rejects_request_above_budget(acc):
    ants = _antennas(acc, 1, seed=24)
    with acc.Server(acc.PRECISION_FP64, lanes=1, hbm_budget_bytes=1 << 20) as srv:
        with pytest.raises(acc.AccelError) as e:
            srv.submit(ants[0])
        assert e.value.code == acc.ERR_TOO_LARGE


@pytest.mark.parametrize("precision", [0, 1])
def test_request_footprint_bounds_the_batch(acc, precision):
    """The admission estimate is an upper bound of what a batch allocates."""
    ants = _antennas(acc, 6, seed=25, n_cap=1500)
    with acc.Server(precision, lanes=1) as srv:
        for a in ants:
            est = srv.shape(a).device_bytes
            b = acc.HallenBatch([a], precision=precision)
            assert b.info.device_bytes <= est, (b.info.device_bytes, est)
            b.close()


def test_server_maps_its_budget_up_front(acc):
    """Creating a server maps its HBM budget into the device's pool, so the
    batches it admits suballocate: serving leaves free device memory
    unchanged."""
    import torch

    ants = _antennas(acc, 12, seed=27)
    acc.device_cache_release()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    budget = 2 << 30
    with acc.Server(acc.PRECISION_MIXED, lanes=2, max_batch=4, hbm_budget_bytes=budget) as srv:
        free1, _ = torch.cuda.mem_get_info()
        assert free0 - free1 >= budget // 2, (free0, free1)
        free = []
        for _ in range(2):  # the first pass also loads any kernel not used before
            reqs = [srv.submit(a) for a in ants]
            for r in reqs:
                srv.wait(r)
                assert np.all(np.asarray(r.result()[3]) == 0)
                r.release()
            torch.cuda.synchronize()
            free.append(torch.cuda.mem_get_info()[0])
        assert free[1] == free[0], free
        assert free1 - free[1] < budget // 8, (free1, free)
