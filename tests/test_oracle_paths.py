"""The oracle's degree-2 conductor-path branch against the reference's own
known answers (nec_solver/tests/general_junction.rs).

Pins (CPU only):
  * build_conductor_paths structure: a single wire is one trivial path with
    free ends (0, 20); a collinear end-to-start pair is one trivial path; a
    start-to-start split is one non-trivial path with one 10-segment arm
    reversed and the two tips as free ends; a T junction and a closed
    square loop give None;
  * start_to_start_split_recovers_single_wire: |Z_split - Z_single| < 0.5
    ohm, both through the path solver;
  * bent_inverted_v_matches_nec2c_resistance: |R - 57.7| < 9 ohm, |X| < 60
    ohm, and R = 55.5 ohm to the one decimal the reference quotes for
    its own result.
Plus properties of the restatement: the path solve of a deck whose paths
are all trivial matches the standard solve to rounding, and the CLI
dispatch (Problem) takes the path branch exactly when some path is
non-trivial.
"""
import numpy as np

from oracle import oracle as O

F = 14.2e6


def W(*rows):
    return O.wires_array(rows)


def S(*rows):
    return O.sources_array(rows)


def _path_zin(wires, sources, feed_tag, feed_seg):
    segs = O.build_geometry(wires)
    paths = O.conductor_paths(segs)
    z = O.assemble_z(segs, F)
    rhs, cosv = O.hallen_rhs_paths(segs, F, sources, paths)
    x, _ = O.solve_hallen_paths(z, rhs, cosv, paths)
    idx = [i for i, s in enumerate(segs) if s["tag"] == feed_tag and s["tag_index"] == feed_seg][0]
    return 1.0 / x[idx]


SPLIT = W((1, 26, (0, 0, 0), (0, 0, 5.282), 0.001), (2, 26, (0, 0, 0), (0, 0, -5.282), 0.001))
SINGLE = W((1, 52, (0, 0, -5.282), (0, 0, 5.282), 0.001))
VEE = W((1, 26, (0, 0, 5.0), (4.46, 0, 2.42), 0.001), (2, 26, (0, 0, 5.0), (-4.46, 0, 2.42), 0.001))


def test_single_wire_is_one_trivial_path():
    p = O.conductor_paths(O.build_geometry(W((1, 21, (0, 0, -5), (0, 0, 5), 0.001))))
    assert len(p) == 1 and not p.nontrivial
    assert tuple(p.free_ends[0]) == (0, 20)
    assert np.all(p.sign == 1.0)


def test_collinear_end_to_start_is_one_trivial_path():
    p = O.conductor_paths(O.build_geometry(W((1, 10, (0, 0, -5), (0, 0, 0), 0.001),
                                             (2, 10, (0, 0, 0), (0, 0, 5), 0.001))))
    assert len(p) == 1 and not p.nontrivial


def test_start_to_start_is_one_nontrivial_path():
    p = O.conductor_paths(O.build_geometry(W((1, 10, (0, 0, 0), (0, 0, 5), 0.001),
                                             (2, 10, (0, 0, 0), (0, 0, -5), 0.001))))
    assert len(p) == 1 and p.nontrivial
    assert int((p.sign < 0).sum()) == 10
    assert tuple(sorted(p.free_ends[0])) == (9, 19)
    # signed arc length runs from -5 to 5 through the join, centred at 0
    order = p.segs(0)
    assert np.all(np.diff(p.s_mid[order]) > 0)
    assert abs(p.s_mid[order].sum()) < 1e-12


def test_t_junction_and_closed_loop_are_unsupported():
    tee = W((1, 5, (0, 0, 0), (5, 0, 0), 0.001), (2, 5, (0, 0, 0), (-5, 0, 0), 0.001),
            (3, 5, (0, 0, 0), (0, 0, 5), 0.001))
    assert O.conductor_paths(O.build_geometry(tee)) is None
    h, s = 2.639, 5.278
    loop = W((1, 6, (-h, 0, 0), (h, 0, 0), 0.001), (2, 6, (h, 0, 0), (h, 0, s), 0.001),
             (3, 6, (h, 0, s), (-h, 0, s), 0.001), (4, 6, (-h, 0, s), (-h, 0, 0), 0.001))
    assert O.conductor_paths(O.build_geometry(loop)) is None


def test_start_to_start_split_recovers_single_wire():
    z_single = _path_zin(SINGLE, S((1, 27, 1.0)), 1, 27)
    z_split = _path_zin(SPLIT, S((1, 1, 1.0)), 1, 1)
    assert z_split.real > 0.0
    assert abs(z_split - z_single) < 0.5


def test_bent_inverted_v_matches_nec2c_resistance():
    z = _path_zin(VEE, S((1, 1, 1.0)), 1, 1)
    assert abs(z.real - 57.7) < 9.0
    assert abs(z.imag) < 60.0
    assert round(z.real, 1) == 55.5


def test_trivial_paths_match_the_standard_solve():
    segs = O.build_geometry(SINGLE)
    paths = O.conductor_paths(segs)
    z = O.assemble_z(segs, F)
    rhs_p, cos_p = O.hallen_rhs_paths(segs, F, S((1, 27, 1.0)), paths)
    rhs_s, cos_s = O.hallen_rhs(segs, F, S((1, 27, 1.0)))
    assert np.abs(cos_p - cos_s).max() < 1e-14
    assert np.abs(rhs_p - rhs_s).max() < 1e-14 * np.abs(rhs_s).max()
    xp, _ = O.solve_hallen_paths(z, rhs_p, cos_p, paths)
    xs, _ = O.solve_hallen(z, rhs_s, cos_s, O.merge_collinear(segs), [], [], [])
    assert abs(1 / xp[26] - 1 / xs[26]) < 1e-9 * abs(1 / xs[26])


def test_problem_dispatch_takes_the_path_branch():
    p = O.Problem(SPLIT, S((1, 1, 1.0)), F)
    O.solve_problem(p)
    assert p.status == 0
    assert p.zin[0] == _path_zin(SPLIT, S((1, 1, 1.0)), 1, 1)
    # a start-to-start split fed on the reversed arm keeps V/I positive
    p2 = O.Problem(SPLIT, S((2, 1, 1.0)), F)
    O.solve_problem(p2)
    assert p2.zin[0].real > 0 and abs(p2.zin[0] - p.zin[0]) < 1e-9 * abs(p.zin[0])
