"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle is a C restatement of the reference CPU Hallen path
(crates/nec_solver/src/{geometry,excitation,matrix,linear,farfield}.rs and
apps/nec-cli/src/solve_session.rs); see fnec_oracle.c for per-function
citations.  Only tests/, __graft_entry__.smoke() and bench.py's CPU arms
import this module.  It is the checker, never the measured product.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

SEG_DTYPE = np.dtype(
    [
        ("tag", "<u4"),
        ("tag_index", "<u4"),
        ("start", "<f8", 3),
        ("end", "<f8", 3),
        ("mid", "<f8", 3),
        ("dir", "<f8", 3),
        ("length", "<f8"),
        ("radius", "<f8"),
    ]
)
WIRE_DTYPE = np.dtype(
    [("tag", "<u4"), ("segments", "<u4"), ("start", "<f8", 3), ("end", "<f8", 3), ("radius", "<f8")]
)
SOURCE_DTYPE = np.dtype([("tag", "<u4"), ("segment", "<u4"), ("v_re", "<f8"), ("v_im", "<f8")])

GROUND_FREE = 0
GROUND_PEC = 1

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double


class _Problem(ctypes.Structure):
    _fields_ = [
        ("wires", _P),
        ("n_wires", _I64),
        ("sources", _P),
        ("n_sources", _I64),
        ("ground", ctypes.c_int),
        ("freq_hz", _D),
        ("points", _P),
        ("n_points", _I64),
        ("currents", _P),
        ("feed", _P),
        ("n_feed", _P),
        ("pattern", _P),
        ("pivots", _P),
        ("status", ctypes.c_int),
        ("loads", _P),
        ("n_loads", _I64),
        ("tls", _P),
        ("n_tls", _I64),
        ("nts", _P),
        ("n_nts", _I64),
        ("wave", _P),
    ]


class _Wave(ctypes.Structure):
    _fields_ = [("ex_type", ctypes.c_int32), ("theta_deg", _D), ("phi_deg", _D), ("eta_deg", _D),
                ("axial_ratio", _D)]


TL_DTYPE = np.dtype([("tag1", np.uint32), ("seg1", np.uint32), ("tag2", np.uint32), ("seg2", np.uint32),
                     ("num_segments", np.uint32), ("tl_type", np.uint32), ("z0", np.float64),
                     ("length", np.float64), ("f3", np.float64)])
NT_DTYPE = np.dtype([("tag1", np.uint32), ("seg1", np.uint32), ("tag2", np.uint32), ("seg2", np.uint32),
                     ("y11r", np.float64), ("y11i", np.float64), ("y12r", np.float64), ("y12i", np.float64),
                     ("y22r", np.float64), ("y22i", np.float64)])


def tls_array(tls) -> np.ndarray:
    """TL cards (tag1, seg1, tag2, seg2, num_segments, tl_type, z0, length, f3)."""
    arr = np.zeros(len(tls), dtype=TL_DTYPE)
    for i, t in enumerate(tls):
        arr[i] = tuple(t)
    return arr


def nts_array(nts) -> np.ndarray:
    """NT cards (tag1, seg1, tag2, seg2, y11r, y11i, y12r, y12i, y22r, y22i)."""
    arr = np.zeros(len(nts), dtype=NT_DTYPE)
    for i, t in enumerate(nts):
        arr[i] = tuple(t)
    return arr


LOAD_DTYPE = np.dtype([("load_type", np.int32), ("tag", np.uint32), ("seg_first", np.uint32),
                       ("seg_last", np.uint32), ("f1", np.float64), ("f2", np.float64), ("f3", np.float64)])


def loads_array(loads) -> np.ndarray:
    """loads: iterable of LD cards (type, tag, seg_first, seg_last, f1, f2, f3)."""
    arr = np.zeros(len(loads), dtype=LOAD_DTYPE)
    for i, (t, tag, s0, s1, f1, f2, f3) in enumerate(loads):
        arr[i] = (t, tag, s0, s1, f1, f2, f3)
    return arr


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, no GPU)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.or_build_geometry.restype = _I64
        L.or_build_geometry.argtypes = [_P, _I64, _P, _I64]
        L.or_wire_endpoints.restype = _I64
        L.or_wire_endpoints.argtypes = [_P, _I64, _P, _I64]
        L.or_merge_collinear.restype = _I64
        L.or_merge_collinear.argtypes = [_P, _I64, _P, _I64]
        L.or_detect_junctions.restype = _I64
        L.or_detect_junctions.argtypes = [_P, _P, _I64, _D, _P, _P, _P, _I64]
        L.or_cli_junctions.restype = _I64
        L.or_cli_junctions.argtypes = [_P, _I64, _P, _I64, _P, _P, _P, _I64]
        L.or_hallen_rhs.restype = ctypes.c_int
        L.or_hallen_rhs.argtypes = [_P, _I64, _D, _P, _I64, _P, _P]
        L.or_excitation.restype = ctypes.c_int
        L.or_excitation.argtypes = [_P, _I64, _P, _I64, _P]
        L.or_assemble_z.restype = None
        L.or_assemble_z.argtypes = [_P, _I64, _D, ctypes.c_int, _P]
        L.or_solve_hallen.restype = ctypes.c_int
        L.or_solve_hallen.argtypes = [_P, _I64, _P, _P, _P, _I64, _P, _P, _P, _I64, _P, _P, _P,
                                      ctypes.c_int, ctypes.c_int]
        L.or_conductor_paths.restype = _I64
        L.or_conductor_paths.argtypes = [_P, _I64, _P, _P, _P, _P, _P]
        L.or_hallen_rhs_paths.restype = ctypes.c_int
        L.or_hallen_rhs_paths.argtypes = [_P, _I64, _D, _P, _I64, _P, _P, _P, _P, _P]
        L.or_solve_hallen_paths.restype = ctypes.c_int
        L.or_solve_hallen_paths.argtypes = [_P, _I64, _P, _P, _P, _P, _I64, _P, _P, _P, ctypes.c_int,
                                            ctypes.c_int]
        L.or_build_loads.restype = _I64
        L.or_build_loads.argtypes = [_P, _I64, _D, _P, _I64, _P]
        L.or_planewave_rhs.restype = ctypes.c_int
        L.or_planewave_rhs.argtypes = [_P, _I64, _D, _P, _P, _P, _P, _P, _P, _P]
        L.or_solve_hallen_planewave.restype = ctypes.c_int
        L.or_solve_hallen_planewave.argtypes = [_P, _I64, _P, _P, _P, _P, _I64, _P, _I64, _P, _P, _P, ctypes.c_int]
        L.or_tl_stamps.restype = _I64
        L.or_tl_stamps.argtypes = [_P, _I64, _D, _P, _I64, _P, _P, _P, _I64]
        L.or_nt_stamps.restype = _I64
        L.or_nt_stamps.argtypes = [_P, _I64, _P, _I64, _P, _P, _P, _I64]
        L.or_near_field.restype = None
        L.or_near_field.argtypes = [_P, _I64, _P, _D, _P, _I64, _P, _P]
        L.or_near_field_points.restype = _I64
        L.or_near_field_points.argtypes = [ctypes.c_uint32] * 4 + [_D] * 6 + [_P]
        L.or_solve_square.restype = ctypes.c_int
        L.or_solve_square.argtypes = [_P, _P, _I64, _P, _P, ctypes.c_int]
        L.or_feedpoints.restype = _I64
        L.or_feedpoints.argtypes = [_P, _I64, _P, _I64, _P, _P, _I64]
        L.or_integrate_power.restype = _D
        L.or_integrate_power.argtypes = [_P, _I64, _P, _D, ctypes.c_int]
        L.or_radiation_pattern.restype = None
        L.or_radiation_pattern.argtypes = [_P, _I64, _P, _D, ctypes.c_int, _P, _I64, _P, _P, _P]
        L.or_rp_card_points.restype = _I64
        L.or_rp_card_points.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _D, _D, _D, _D, _P]
        L.or_solve_problem.restype = ctypes.c_int
        L.or_solve_problem.argtypes = [_P]
        L.or_solve_problems.restype = None
        L.or_solve_problems.argtypes = [_P, _I64, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def wires_array(wires) -> np.ndarray:
    """wires: iterable of (tag, segments, start3, end3, radius)."""
    arr = np.zeros(len(wires), dtype=WIRE_DTYPE)
    for i, (tag, nseg, s, e, r) in enumerate(wires):
        arr[i] = (tag, nseg, s, e, r)
    return arr


def sources_array(sources) -> np.ndarray:
    """sources: iterable of (tag, segment, v_complex)."""
    arr = np.zeros(len(sources), dtype=SOURCE_DTYPE)
    for i, (tag, seg, v) in enumerate(sources):
        arr[i] = (tag, seg, complex(v).real, complex(v).imag)
    return arr


class OracleError(RuntimeError):
    pass


def build_geometry(wires: np.ndarray) -> np.ndarray:
    cap = int(wires["segments"].sum())
    out = np.zeros(max(cap, 1), dtype=SEG_DTYPE)
    n = lib().or_build_geometry(_ptr(wires), len(wires), _ptr(out), cap)
    if n < 0:
        raise OracleError(f"build_geometry: status {n}")
    return out[:n]


def wire_endpoints(segs: np.ndarray) -> np.ndarray:
    cnt = lib().or_wire_endpoints(_ptr(segs), len(segs), None, 0)
    out = np.zeros((max(cnt, 1), 2), dtype=np.int64)
    lib().or_wire_endpoints(_ptr(segs), len(segs), _ptr(out), cnt)
    return out[:cnt]


def merge_collinear(segs: np.ndarray) -> np.ndarray:
    cnt = lib().or_merge_collinear(_ptr(segs), len(segs), None, 0)
    out = np.zeros((max(cnt, 1), 2), dtype=np.int64)
    lib().or_merge_collinear(_ptr(segs), len(segs), _ptr(out), cnt)
    return out[:cnt]


def detect_junctions(segs, endpoints, tol=1e-6):
    ep = np.ascontiguousarray(endpoints, dtype=np.int64)
    cnt = lib().or_detect_junctions(_ptr(segs), _ptr(ep), len(ep), tol, None, None, None, 0)
    a = np.zeros(max(cnt, 1), np.int64)
    b = np.zeros(max(cnt, 1), np.int64)
    s = np.zeros(max(cnt, 1), np.float64)
    lib().or_detect_junctions(_ptr(segs), _ptr(ep), len(ep), tol, _ptr(a), _ptr(b), _ptr(s), cnt)
    return a[:cnt], b[:cnt], s[:cnt]


def cli_junctions(segs, merged):
    ep = np.ascontiguousarray(merged, dtype=np.int64)
    cnt = lib().or_cli_junctions(_ptr(segs), len(segs), _ptr(ep), len(ep), None, None, None, 0)
    a = np.zeros(max(cnt, 1), np.int64)
    b = np.zeros(max(cnt, 1), np.int64)
    s = np.zeros(max(cnt, 1), np.float64)
    lib().or_cli_junctions(_ptr(segs), len(segs), _ptr(ep), len(ep), _ptr(a), _ptr(b), _ptr(s), cnt)
    return a[:cnt], b[:cnt], s[:cnt]


def hallen_rhs(segs, freq_hz, sources):
    n = len(segs)
    rhs = np.zeros(n, np.complex128)
    cosv = np.zeros(n, np.float64)
    st = lib().or_hallen_rhs(_ptr(segs), n, freq_hz, _ptr(sources), len(sources), _ptr(rhs), _ptr(cosv))
    if st != 0:
        raise OracleError(f"hallen_rhs: status {st}")
    return rhs, cosv


def excitation(segs, sources):
    v = np.zeros(len(segs), np.complex128)
    st = lib().or_excitation(_ptr(segs), len(segs), _ptr(sources), len(sources), _ptr(v))
    if st != 0:
        raise OracleError(f"excitation: status {st}")
    return v


def assemble_z(segs, freq_hz, ground=GROUND_FREE):
    n = len(segs)
    z = np.zeros((n, n), np.complex128)
    lib().or_assemble_z(_ptr(segs), n, freq_hz, ground, _ptr(z))
    return z


def solve_hallen(z, rhs, cosv, endpoints, ja, jb, js, naive=False, want_gram=False, nthreads=1):
    n = z.shape[0]
    z = np.ascontiguousarray(z, np.complex128)
    rhs = np.ascontiguousarray(rhs, np.complex128)
    cosv = np.ascontiguousarray(cosv, np.float64)
    ep = np.ascontiguousarray(endpoints, np.int64).reshape(-1, 2)
    w = len(ep) if (len(ep) > 0 and n > 0) else (1 if n > 0 else 0)
    ja = np.ascontiguousarray(ja, np.int64)
    jb = np.ascontiguousarray(jb, np.int64)
    js = np.ascontiguousarray(js, np.float64)
    s = n + w
    x = np.zeros(s, np.complex128)
    piv = np.zeros(max(s, 1), np.int32)
    gram = np.zeros((s, s + 1), np.complex128) if want_gram else None
    st = lib().or_solve_hallen(_ptr(z), n, _ptr(rhs), _ptr(cosv), _ptr(ep), len(ep), _ptr(ja), _ptr(jb),
                               _ptr(js), len(ja), _ptr(x), _ptr(piv), _ptr(gram), int(naive), nthreads)
    if st != 0:
        raise OracleError(f"solve_hallen: status {st}")
    return (x, piv[:s], gram) if want_gram else (x, piv[:s])


class ConductorPaths:
    """build_conductor_paths (geometry.rs:404-584) for a segment list:
    per-segment path index, traversal sign and signed arc length, the free
    ends (2 per path) and whether some path is non-trivial."""

    def __init__(self, path_of, sign, s_mid, free_ends, nontrivial):
        self.path_of, self.sign, self.s_mid = path_of, sign, s_mid
        self.free_ends = free_ends
        self.nontrivial = nontrivial

    def __len__(self):
        return len(self.free_ends)

    def segs(self, p):
        """Segments of path p in traversal order (signed arc length ascending)."""
        idx = np.nonzero(self.path_of == p)[0]
        return idx[np.argsort(self.s_mid[idx], kind="stable")]


def conductor_paths(segs):
    """ConductorPaths, or None where the reference returns None."""
    n = len(segs)
    path_of = np.zeros(max(n, 1), np.int64)
    sign = np.zeros(max(n, 1), np.float64)
    s_mid = np.zeros(max(n, 1), np.float64)
    fe = np.zeros((max(n, 1), 2), np.int64)
    nt = ctypes.c_int(0)
    cnt = lib().or_conductor_paths(_ptr(segs), n, _ptr(path_of), _ptr(sign), _ptr(s_mid), _ptr(fe), ctypes.byref(nt))
    if cnt < 0:
        return None
    return ConductorPaths(path_of[:n], sign[:n], s_mid[:n], fe[:cnt], bool(nt.value))


def hallen_rhs_paths(segs, freq_hz, sources, paths: ConductorPaths):
    n = len(segs)
    rhs = np.zeros(n, np.complex128)
    cosv = np.zeros(n, np.float64)
    st = lib().or_hallen_rhs_paths(_ptr(segs), n, freq_hz, _ptr(sources), len(sources), _ptr(paths.path_of),
                                   _ptr(paths.sign), _ptr(paths.s_mid), _ptr(rhs), _ptr(cosv))
    if st != 0:
        raise OracleError(f"hallen_rhs_paths: status {st}")
    return rhs, cosv


def solve_hallen_paths(z, rhs, cosv, paths: ConductorPaths, nthreads=1):
    n = z.shape[0]
    z = np.ascontiguousarray(z, np.complex128)
    rhs = np.ascontiguousarray(rhs, np.complex128)
    cosv = np.ascontiguousarray(cosv, np.float64)
    fe = np.ascontiguousarray(paths.free_ends, np.int64).reshape(-1)
    s = n + len(paths)
    x = np.zeros(s, np.complex128)
    piv = np.zeros(max(s, 1), np.int32)
    st = lib().or_solve_hallen_paths(_ptr(z), n, _ptr(rhs), _ptr(cosv), _ptr(paths.path_of), _ptr(fe), len(fe),
                                     _ptr(x), _ptr(piv), None, 0, nthreads)
    if st != 0:
        raise OracleError(f"solve_hallen_paths: status {st}")
    return x, piv[:s]


def wave(ex_type=1, theta_deg=0.0, phi_deg=0.0, eta_deg=0.0, axial_ratio=0.0):
    """One incident plane wave (planewave.rs IncidentPlaneWave): EX type
    1 linear, 2 right / 3 left elliptic."""
    return _Wave(int(ex_type), float(theta_deg), float(phi_deg), float(eta_deg), float(axial_ratio))


def planewave_rhs(segs, freq_hz, w, paths=None):
    """planewave.rs build_planewave_hallen (paths None) or
    build_planewave_hallen_paths: (rhs, cos_vec, sin_vec)."""
    n = len(segs)
    rhs = np.zeros(n, np.complex128)
    cosv = np.zeros(n, np.float64)
    sinv = np.zeros(n, np.float64)
    args = (None, None, None) if paths is None else (_ptr(paths.path_of), _ptr(paths.sign), _ptr(paths.s_mid))
    st = lib().or_planewave_rhs(_ptr(segs), n, float(freq_hz), ctypes.byref(w), *args, _ptr(rhs), _ptr(cosv),
                                _ptr(sinv))
    if st != 0:
        raise OracleError(f"planewave_rhs: status {st}")
    return rhs, cosv, sinv


def solve_hallen_planewave(z, rhs, cosv, sinv, row_wire, n_cols, free_ends=None, naive=False):
    """linear.rs solve_hallen_planewave (free_ends None: both ends of every
    per-tag wire) / solve_hallen_planewave_paths: (x, pivots, gram)."""
    n = z.shape[0]
    z = np.ascontiguousarray(z, np.complex128)
    s = n + 2 * n_cols
    x = np.zeros(s, np.complex128)
    piv = np.zeros(max(s, 1), np.int32)
    gram = np.zeros((s, s + 1), np.complex128)
    rw = np.ascontiguousarray(row_wire, np.int64)
    fe = None if free_ends is None else np.ascontiguousarray(free_ends, np.int64).reshape(-1)
    st = lib().or_solve_hallen_planewave(_ptr(z), n, _ptr(np.ascontiguousarray(rhs, np.complex128)),
                                         _ptr(np.ascontiguousarray(cosv, np.float64)),
                                         _ptr(np.ascontiguousarray(sinv, np.float64)), _ptr(rw), int(n_cols),
                                         _ptr(fe), 0 if fe is None else len(fe), _ptr(x), _ptr(piv), _ptr(gram),
                                         int(bool(naive)))
    if st != 0:
        raise OracleError(f"solve_hallen_planewave: status {st}")
    return x, piv[:s], gram


def wave_directions(ex_type, n_theta, n_phi, theta0, phi0, d_theta, d_phi, eta_deg=0.0, axial_ratio=0.0):
    """solve_session.rs:313-355: the incidence grid of one plane-wave EX card,
    theta outer, phi inner; the first is the deck's own direction."""
    out = []
    for it in range(max(int(n_theta), 1)):
        for ip in range(max(int(n_phi), 1)):
            out.append(wave(ex_type, theta0 + it * float(d_theta), phi0 + ip * float(d_phi), eta_deg, axial_ratio))
    return out


def receive_sweep(wires, freq_hz, waves, ground=GROUND_FREE, loads=None, tls=None, nts=None):
    """solve_session.rs:313-375 plane_wave_receive_sweep: one full receive
    solve per incidence direction, the peak |I| of each, and the response
    20 log10(peak / max peak) dB (-999.99 for a zero peak).  Returns
    (peaks, response_db, currents of every direction)."""
    peaks, cur = [], []
    for w in waves:
        p = solve_problem(Problem(wires, sources_array([]), freq_hz, ground=ground, loads=loads, tls=tls, nts=nts,
                                  wave=w))
        if p.status != 0:
            raise OracleError(f"receive solve: status {p.status}")
        mags = [math.hypot(c.real, c.imag) for c in p.currents]
        peaks.append(max([0.0] + mags))
        cur.append(p.currents.copy())
    top = max([0.0] + peaks)
    db = [20.0 * math.log10(pk / top) if pk > 0.0 and top > 0.0 else -999.99 for pk in peaks]
    return np.array(peaks), np.array(db), cur


def build_loads(segs, freq_hz, loads):
    """loads.rs build_loads: (per-segment load impedance, ignored count)."""
    n = len(segs)
    out = np.zeros(max(n, 1), np.complex128)
    ld = np.ascontiguousarray(loads, LOAD_DTYPE)
    ign = lib().or_build_loads(_ptr(segs), n, float(freq_hz), _ptr(ld), len(ld), _ptr(out))
    return out[:n], int(ign)


def tl_stamps(segs, freq_hz, tls):
    """tl.rs build_tl_stamps: [(row, col, delta)] in order."""
    t = np.ascontiguousarray(tls, TL_DTYPE)
    cap = 4 * len(t) + 1
    r, c, v = np.zeros(cap, np.int64), np.zeros(cap, np.int64), np.zeros(cap, np.complex128)
    k = lib().or_tl_stamps(_ptr(segs), len(segs), float(freq_hz), _ptr(t), len(t), _ptr(r), _ptr(c), _ptr(v), cap)
    return list(zip(r[:k].tolist(), c[:k].tolist(), v[:k].tolist()))


def nt_stamps(segs, nts):
    """network.rs build_nt_stamps: [(row, col, delta)] in order."""
    t = np.ascontiguousarray(nts, NT_DTYPE)
    cap = 4 * len(t) + 1
    r, c, v = np.zeros(cap, np.int64), np.zeros(cap, np.int64), np.zeros(cap, np.complex128)
    k = lib().or_nt_stamps(_ptr(segs), len(segs), _ptr(t), len(t), _ptr(r), _ptr(c), _ptr(v), cap)
    return list(zip(r[:k].tolist(), c[:k].tolist(), v[:k].tolist()))


def near_field(segs, currents, freq_hz, points):
    """farfield.rs near_e_field / near_h_field: (E, H), each (p, 3) complex."""
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    cur = np.ascontiguousarray(currents, np.complex128)
    e = np.zeros((max(len(pts), 1), 3), np.complex128)
    h = np.zeros((max(len(pts), 1), 3), np.complex128)
    lib().or_near_field(_ptr(segs), len(segs), _ptr(cur), float(freq_hz), _ptr(pts), len(pts), _ptr(e), _ptr(h))
    return e[: len(pts)], h[: len(pts)]


def near_field_points(coord_type, nx, ny, nz, x0, y0, z0, dx, dy, dz):
    """The observation points of one NE/NH card, (p, 3)."""
    args = [int(coord_type), int(nx), int(ny), int(nz)] + [float(v) for v in (x0, y0, z0, dx, dy, dz)]
    cnt = lib().or_near_field_points(*args, None)
    out = np.zeros((max(cnt, 1), 3), np.float64)
    lib().or_near_field_points(*args, _ptr(out))
    return out[:cnt]


def solve_square(a, b, nthreads=1):
    s = a.shape[0]
    a = np.array(a, np.complex128, order="C")
    b = np.array(b, np.complex128)
    x = np.zeros(s, np.complex128)
    piv = np.zeros(max(s, 1), np.int32)
    st = lib().or_solve_square(_ptr(a), _ptr(b), s, _ptr(x), _ptr(piv), nthreads)
    return st, x, piv[:s]


def feedpoints(segs, sources, currents):
    out = np.zeros((max(len(sources), 1), 7), np.float64)
    cur = np.ascontiguousarray(currents, np.complex128)
    cnt = lib().or_feedpoints(_ptr(segs), len(segs), _ptr(sources), len(sources), _ptr(cur), _ptr(out),
                              len(sources))
    return out[:cnt]


def integrate_power(segs, currents, freq_hz, ground=GROUND_FREE):
    cur = np.ascontiguousarray(currents, np.complex128)
    return lib().or_integrate_power(_ptr(segs), len(segs), _ptr(cur), freq_hz, ground)


def radiation_pattern(segs, currents, freq_hz, points, ground=GROUND_FREE, want_fields=False):
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 2)
    cur = np.ascontiguousarray(currents, np.complex128)
    out = np.zeros((len(pts), 4), np.float64)
    tot = np.zeros(1, np.float64)
    uf = np.zeros((len(pts), 2), np.complex128) if want_fields else None
    lib().or_radiation_pattern(_ptr(segs), len(segs), _ptr(cur), freq_hz, ground, _ptr(pts), len(pts),
                               _ptr(out), _ptr(tot), _ptr(uf))
    if want_fields:
        return out, float(tot[0]), uf
    return out, float(tot[0])


def rp_card_points(n_theta, n_phi, theta0, phi0, d_theta, d_phi):
    cnt = lib().or_rp_card_points(n_theta, n_phi, theta0, phi0, d_theta, d_phi, None)
    pts = np.zeros((cnt, 2), np.float64)
    lib().or_rp_card_points(n_theta, n_phi, theta0, phi0, d_theta, d_phi, _ptr(pts))
    return pts


class Problem:
    """One per-frequency CLI Hallen solve (solve_session.rs:1186-1437): the
    degree-2 conductor-path branch when some path is non-trivial
    (:1338-1378), else the standard branch."""

    def __init__(self, wires, sources, freq_hz, ground=GROUND_FREE, points=None, loads=None, tls=None, nts=None,
                 wave=None):
        self.wave = wave
        self.loads = None if loads is None or len(loads) == 0 else np.ascontiguousarray(loads, LOAD_DTYPE)
        self.tls = None if tls is None or len(tls) == 0 else np.ascontiguousarray(tls, TL_DTYPE)
        self.nts = None if nts is None or len(nts) == 0 else np.ascontiguousarray(nts, NT_DTYPE)
        self.wires = np.ascontiguousarray(wires)
        self.sources = np.ascontiguousarray(sources)
        self.freq_hz = float(freq_hz)
        self.ground = int(ground)
        self.points = None if points is None else np.ascontiguousarray(points, np.float64).reshape(-1, 2)
        n = int(self.wires["segments"].sum())
        w = len(self.wires)
        self.currents = np.zeros(n, np.complex128)
        self.feed = np.zeros((max(len(self.sources), 1), 7), np.float64)
        self.n_feed = np.zeros(1, np.int64)
        npts = 0 if self.points is None else len(self.points)
        self.pattern = np.zeros((max(npts, 1), 4), np.float64)
        self.pivots = np.zeros(n + 2 * w, np.int32)
        self._s = _Problem(
            _ptr(self.wires), len(self.wires), _ptr(self.sources), len(self.sources), self.ground,
            self.freq_hz, _ptr(self.points), npts, _ptr(self.currents), _ptr(self.feed),
            _ptr(self.n_feed), _ptr(self.pattern), _ptr(self.pivots), 0, _ptr(self.loads),
            0 if self.loads is None else len(self.loads), _ptr(self.tls), 0 if self.tls is None else len(self.tls),
            _ptr(self.nts), 0 if self.nts is None else len(self.nts),
            None if wave is None else ctypes.addressof(wave))

    @property
    def status(self):
        return self._s.status

    @property
    def zin(self):
        f = self.feed[: int(self.n_feed[0])]
        return f[:, 5] + 1j * f[:, 6]


def solve_problem(p: Problem) -> Problem:
    lib().or_solve_problem(ctypes.byref(p._s))
    return p


def solve_problems(problems, nthreads: int):
    arr = (_Problem * len(problems))(*[p._s for p in problems])
    lib().or_solve_problems(ctypes.cast(arr, _P), len(problems), int(nthreads))
    for i, p in enumerate(problems):
        p._s = arr[i]
    return problems
