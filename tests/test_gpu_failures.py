"""Failure paths, made on purpose without faulting, trapping or hanging the GPU.

Every device wait in the library is bounded (the grid barrier of the
cooperative panel and refinement kernels, the tcgen05 GEMM's mbarrier
waits): when one runs out, the kernel marks the unit FNEC_UNIT_TIMEOUT,
drains what it has in flight and returns, so the context stays usable.
These tests make such waits run out with a short limit (a CTA that never
arrives, a GEMM whose loads stop), inject a device allocation failure on the
host, and hand the library non-finite geometry, then check that the error is
reported where it belongs and that the next call works.  The reference's own
error path is the singular pivot (linear.rs:1354), tested elsewhere.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

DIPOLE = [(1, 51, (0.0, 0.0, -5.282), (0.0, 0.0, 5.282), 0.001)]


@pytest.fixture(scope="module")
def acc():
    import nec_accel

    nec_accel.default_context()
    return nec_accel


def _dipole_ok(acc):
    """A small solve after a failure: still the oracle's answer bit for bit."""
    ant = acc.Antenna(acc.wires_array(DIPOLE), acc.sources_array([(1, 26, 1.0)]), [14.2e6], acc.GROUND_FREE, None)
    batch = acc.HallenBatch([ant])
    res = batch.solve()
    p = O.Problem(O.wires_array(DIPOLE), O.sources_array([(1, 26, 1.0)]), 14.2e6)
    O.solve_problem(p)
    assert res.status[0] == 0
    assert np.array_equal(res.currents[0].view(np.uint64), p.currents.view(np.uint64))
    batch.close()


def test_grid_barrier_gives_up_when_a_cta_never_arrives(acc):
    """A cooperative launch whose CTA 3 of 8 never reaches the barrier: the
    other seven wait 1 ms, mark FNEC_UNIT_TIMEOUT and return."""
    st, ms = acc.selftest_wait_timeout(acc.WAIT_GRID_ABSENT_CTA, wait_ns=1_000_000)
    assert st == acc.UNIT_TIMEOUT
    assert 0.9 <= ms < 1000.0, ms
    st, ms = acc.selftest_wait_timeout(acc.WAIT_GRID_ALL_ARRIVE, wait_ns=1_000_000)
    assert st == 0
    assert ms < 100.0
    _dipole_ok(acc)


def test_gemm_wait_runs_out_drains_and_frees_tmem(acc):
    """The tcgen05 GEMM with its loads stopped after 2 of 8 k-blocks: the MMA
    warp's wait runs out after 1 ms, the CTA lets its two issued k-blocks'
    copies and MMAs complete, frees its TMEM and marks the status.  TMEM
    really was freed: the regular GEMM then runs (every CTA allocates TMEM)
    and is right."""
    for _ in range(3):
        st, ms = acc.selftest_wait_timeout(acc.WAIT_GEMM_LOADS_STOPPED, wait_ns=1_000_000)
        assert st == acc.UNIT_TIMEOUT
    rng = np.random.default_rng(4)
    a = rng.standard_normal((300, 96)).astype(np.float32)
    b = rng.standard_normal((200, 96)).astype(np.float32)
    c = acc.selftest_tf32x3_gemm(a, b)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    assert np.abs(c - ref).max() <= 1e-4 * np.abs(ref).max()
    _dipole_ok(acc)


@pytest.mark.parametrize("after", [0, 3, 9])
def test_device_allocation_failure_is_reported_and_leaks_nothing(acc, after):
    """The after-th device allocation of a batch fails as if the GPU were
    full: batch creation returns OUT_OF_MEMORY, frees what it had taken,
    and the next batch works."""
    import torch

    ant = acc.Antenna(acc.wires_array(DIPOLE), acc.sources_array([(1, 26, 1.0)]), [14.2e6, 14.5e6],
                      acc.GROUND_PEC, (19, 1, 0.0, 0.0, 5.0, 0.0))
    for prec in (acc.PRECISION_FP64, acc.PRECISION_MIXED):
        warm = acc.HallenBatch([ant], precision=prec)  # first-use allocations (module, pools) happen here
        warm.solve()
        warm.close()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        acc.test_fail_device_allocation(after)
        try:
            with pytest.raises(acc.AccelError) as ei:
                acc.HallenBatch([ant], precision=prec)
            assert ei.value.code == acc.ERR_OUT_OF_MEMORY
        finally:
            acc.test_fail_device_allocation(-1)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
    _dipole_ok(acc)


def test_freed_batch_memory_is_reused_then_released(acc):
    """A destroyed batch's device memory stays in the stream-ordered pool: a
    second batch of the same shape takes it without growing the pool, and
    device_cache_release hands it back to the driver; page-locked blocks are
    kept the same way until host_cache_release."""
    import torch

    ant = acc.Antenna(acc.wires_array(DIPOLE), acc.sources_array([(1, 26, 1.0)]),
                      [14.0e6 + 0.1e6 * k for k in range(64)], acc.GROUND_FREE, (19, 37, 0.0, 5.0, 0.0, 10.0))
    for prec in (acc.PRECISION_FP64, acc.PRECISION_MIXED):
        b = acc.HallenBatch([ant] * 8, precision=prec)
        ref = np.concatenate(b.solve().currents)
        b.close()
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        b = acc.HallenBatch([ant] * 8, precision=prec)
        cur = np.concatenate(b.solve().currents)
        assert np.array_equal(cur.view(np.uint64), ref.view(np.uint64))
        b.close()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0
        released = acc.device_cache_release()
        free2, _ = torch.cuda.mem_get_info()
        assert released > 0 and free2 > free1
    assert acc.host_cache_release() > 0
    _dipole_ok(acc)


def test_non_finite_geometry_is_refused_for_that_antenna_only(acc):
    """A NaN coordinate, an infinite radius or a NaN frequency never reaches
    a kernel: a batch naming such an antenna is refused with the antenna's
    index; in the server, only that request is refused while the others
    solve to the same bits as alone."""
    good = [acc.Antenna(acc.wires_array([(1, 21 + 2 * k, (0.0, 0.0, 1.0), (0.0, 0.3 * k, 6.0 + k), 0.001)]),
                        acc.sources_array([(1, 11 + k, 1.0)]), [14.2e6], acc.GROUND_PEC, None) for k in range(4)]
    bad = [acc.Antenna(acc.wires_array([(1, 21, (0.0, np.nan, 1.0), (0.0, 0.0, 6.0), 0.001)]),
                       acc.sources_array([(1, 11, 1.0)]), [14.2e6], acc.GROUND_FREE, None),
           acc.Antenna(acc.wires_array([(1, 21, (0.0, 0.0, 1.0), (0.0, 0.0, 6.0), np.inf)]),
                       acc.sources_array([(1, 11, 1.0)]), [14.2e6], acc.GROUND_FREE, None),
           acc.Antenna(acc.wires_array(DIPOLE), acc.sources_array([(1, 26, 1.0)]), [np.nan], acc.GROUND_FREE, None)]
    for b in bad:
        with pytest.raises(acc.AccelError) as ei:
            acc.HallenBatch(good[:2] + [b] + good[2:])
        assert ei.value.code == acc.ERR_BAD_ARG
        assert "antenna 2" in str(ei.value)
    alone = []
    for g in good:
        bt = acc.HallenBatch([g])
        alone.append(bt.solve().currents[0].copy())
        bt.close()
    with acc.Server(acc.PRECISION_FP64, lanes=2, hbm_budget_bytes=1 << 30) as srv:
        reqs = []
        for k, g in enumerate(good):
            reqs.append(srv.submit(g, tag=k))
            with pytest.raises(acc.AccelError) as ei:
                srv.submit(bad[k % len(bad)])
            assert ei.value.code == acc.ERR_BAD_ARG
        for r in reqs:
            srv.wait(r)
            cur = r.result()[0]
            assert np.array_equal(np.asarray(cur).reshape(-1).view(np.uint64),
                                  alone[r.tag].reshape(-1).view(np.uint64))
            r.release()
