"""The pattern entry point that allocates no device memory.

It exists for callers that cannot call cudaMalloc (a host framework that
owns all device memory through its own pool, a plugin held to a fixed
memory budget, a real-time loop that cannot take cudaMalloc's implicit
synchronisation).  The test gives it caller-owned device buffers (made by
torch here, as such a caller's framework would) and checks two calls in a
row against the allocating entry point fnec_radiation_pattern, within the
gain tolerance of the other parity tests (1e-6 dB; axial ratio 1e-9; the
power integral 1e-12 relative).  The second call uses a different geometry,
ground and point count, so stale scratch from the first would show.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

GAIN_TOL_DB = 1e-6


def _cases():
    # 1) 51-segment dipole over PEC ground, theta cut with below-horizon points
    w1 = O.wires_array([(1, 51, (0, 0, 4.718), (0, 0, 15.282), 1e-3)])
    s1 = O.sources_array([(1, 26, 1.0)])
    p1 = O.Problem(w1, s1, 14.2e6, ground=1)
    O.solve_problem(p1)
    pts1 = O.rp_card_points(37, 2, 0.0, 0.0, 5.0, 90.0)
    # 2) 5-wire array in free space, the full 91 x 361 grid
    rng = np.random.default_rng(11)
    lam = 299792458.0 / 14.2e6
    x, wl = 0.0, []
    for t in range(5):
        L = rng.uniform(0.9, 1.1) * lam / 2
        wl.append((t + 1, 51, (x, 0.0, -L / 2), (x, 0.0, L / 2), 1e-3))
        x += rng.uniform(0.15, 0.25) * lam
    w2 = O.wires_array(wl)
    p2 = O.Problem(w2, O.sources_array([(2, 26, 1.0)]), 14.7e6)
    O.solve_problem(p2)
    pts2 = O.rp_card_points(91, 361, 0.0, 0.0, 1.0, 1.0)
    return [(O.build_geometry(w1), p1.currents, 14.2e6, 1, pts1),
            (O.build_geometry(w2), p2.currents, 14.7e6, 0, pts2)]


def test_noalloc_pattern_matches_allocating_entry_point_twice():
    import torch

    import nec_accel as acc

    dev = torch.device("cuda", 0)
    for segs, cur, f, ground, pts in _cases():
        gseg = acc.gpu_segments_from(segs)
        ref, tot_ref = acc.compute_radiation_pattern(gseg, cur, f, pts, ground)
        d_seg = torch.from_numpy(gseg.view(np.uint8).copy()).to(dev)
        d_cur = torch.from_numpy(np.ascontiguousarray(cur).view(np.float64).copy()).to(dev)
        d_pts = torch.from_numpy(np.ascontiguousarray(pts, np.float64).ravel().copy()).to(dev)
        d_out = torch.full((len(pts) * 4,), np.nan, dtype=torch.float64, device=dev)
        d_tot = torch.zeros(1, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev)
        st = acc.radiation_pattern_noalloc(d_seg.data_ptr(), len(gseg), d_cur.data_ptr(), f, ground,
                                           d_pts.data_ptr(), len(pts), d_out.data_ptr(), d_tot.data_ptr(),
                                           stream.cuda_stream)
        assert st == acc.OK
        torch.cuda.synchronize(dev)
        out = d_out.cpu().numpy().reshape(-1, 4)
        tot = float(d_tot.cpu().numpy()[0])
        assert abs(tot - tot_ref) <= 1e-12 * tot_ref
        clamp = ref[:, 0] <= -999.0
        assert np.array_equal(out[clamp, 0], ref[clamp, 0])
        for col in (0, 1, 2):
            live = ref[:, col] > -999.0
            assert np.abs(out[live, col] - ref[live, col]).max(initial=0.0) <= GAIN_TOL_DB
            assert np.array_equal(out[~live, col], ref[~live, col])
        assert np.abs(out[:, 3] - ref[:, 3]).max() <= 1e-9


def _run_noalloc(acc, torch, dev, gseg, cur, f, ground, pts):
    d_seg = torch.from_numpy(gseg.view(np.uint8).copy()).to(dev)
    d_cur = torch.from_numpy(np.ascontiguousarray(cur).view(np.float64).copy()).to(dev)
    d_pts = torch.from_numpy(np.ascontiguousarray(pts, np.float64).ravel().copy()).to(dev)
    d_out = torch.full((len(pts) * 4,), np.nan, dtype=torch.float64, device=dev)
    d_tot = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def call():
        return acc.radiation_pattern_noalloc(d_seg.data_ptr(), len(gseg), d_cur.data_ptr(), f, ground,
                                             d_pts.data_ptr(), len(pts), d_out.data_ptr(), d_tot.data_ptr(),
                                             stream.cuda_stream)

    return call, d_out, d_tot


@pytest.mark.parametrize("n_wires,seg_per_wire,n_theta,n_phi,ground", [
    (4, 250, 64, 32, 1),      # 1000 segments: runs + currents staged above the default 48 KB
    (8, 512, 256, 256, 0),    # the maxima: 4096 segments (unstaged branch), 65,536 points
])
def test_noalloc_large_cases_allocate_nothing(n_wires, seg_per_wire, n_theta, n_phi, ground):
    """Sizes that take the far field's other shared-memory branches, up to
    the entry point's maxima (4096 segments, 65,536 points), against the
    allocating entry point; after a first call, a call changes the device's
    free memory by nothing (cudaMemGetInfo)."""
    import torch

    import nec_accel as acc

    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(n_wires)
    wl = []
    for t in range(n_wires):
        p0 = rng.uniform([-10, -10, 1], [10, 10, 20])
        p1 = rng.uniform([-10, -10, 1], [10, 10, 20])
        wl.append((t + 1, seg_per_wire, tuple(p0), tuple(p1), 1e-3))
    segs = O.build_geometry(O.wires_array(wl))
    n = len(segs)
    assert n == n_wires * seg_per_wire <= acc.NOALLOC_MAX_SEGMENTS
    cur = rng.normal(size=n) + 1j * rng.normal(size=n)
    pts = O.rp_card_points(n_theta, n_phi, 0.0, 0.0, 90.0 / n_theta if ground else 180.0 / n_theta,
                           360.0 / n_phi)
    assert len(pts) <= acc.NOALLOC_MAX_POINTS
    f = 7.1e6
    gseg = acc.gpu_segments_from(segs)
    ref, tot_ref = acc.compute_radiation_pattern(gseg, cur, f, pts, ground)
    call, d_out, d_tot = _run_noalloc(acc, torch, dev, gseg, cur, f, ground, pts)
    assert call() == acc.OK
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    assert call() == acc.OK
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0
    out = d_out.cpu().numpy().reshape(-1, 4)
    tot = float(d_tot.cpu().numpy()[0])
    assert abs(tot - tot_ref) <= 1e-12 * tot_ref
    for col in (0, 1, 2):
        live = ref[:, col] > -999.0
        assert np.abs(out[live, col] - ref[live, col]).max(initial=0.0) <= GAIN_TOL_DB
        assert np.array_equal(out[~live, col], ref[~live, col])
    assert np.abs(out[:, 3] - ref[:, 3]).max() <= 1e-9


def test_noalloc_rejects_sizes_beyond_its_static_maximum():
    import nec_accel as acc

    # rejected on the host before any device work: the pointers are never used
    st = acc.radiation_pattern_noalloc(1, acc.NOALLOC_MAX_SEGMENTS + 1, 1, 14.2e6, 0, 1, 10, 1)
    assert st == acc.ERR_TOO_LARGE
    st = acc.radiation_pattern_noalloc(1, 10, 1, 14.2e6, 0, 1, acc.NOALLOC_MAX_POINTS + 1, 1)
    assert st == acc.ERR_TOO_LARGE
