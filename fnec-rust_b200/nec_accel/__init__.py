"""Host-side mirror of fnec-rust's ``nec_accel`` crate over libfnec_cuda.so.

The reference's accelerator crate (crates/nec_accel/src/lib.rs:52-96,
wgpu_device.rs) exposes ``fill_zmatrix_wgpu``, ``solve_hallen_gpu_resident``,
``run_rp_farfield_batch_wgpu``, ``microbench_zmatrix_dispatch``,
``enumerate_compute_adapters`` and ``dispatch_frequency_point``.  This module
keeps those names and argument meanings (segments, rhs, cos_vec, wire
endpoints, junctions, frequency) and calls the CUDA library through its C
ABI (include/fnec_cuda.h).  Differences in error behaviour are deliberate:
where the reference returns ``None`` and lets its caller fall back to the
CPU, these functions raise :class:`AccelError` -- there is no CPU fallback.

The batched interface (:class:`HallenBatch`) runs whole per-frequency
solves (solve_session.rs:1186-1437 + the RP grid of :1645) for many
antennas and frequencies in one device pipeline.
"""
from __future__ import annotations

import atexit
import time
import ctypes
import os
import weakref
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfnec_cuda.so")

OK = 0
ERR_BAD_ARG = -1
ERR_NO_DEVICE = -2
ERR_OUT_OF_MEMORY = -3
ERR_CUDA = -4
ERR_SINGULAR = -5
ERR_SEGMENT_NOT_FOUND = -6
ERR_UNSUPPORTED = -7
ERR_TIMEOUT = -8
ERR_BUSY = -9
ERR_TOO_LARGE = -10
NOALLOC_MAX_SEGMENTS = 4096
UNIT_TIMEOUT = 0x40000000  # per-unit status: a bounded device wait gave up
NOALLOC_MAX_POINTS = 65536

GROUND_FREE = 0
GROUND_PEC = 1
PRECISION_FP64 = 0
PRECISION_MIXED = 1

ZSEGMENT_DTYPE = np.dtype([("midpoint", "<f8", 3), ("direction", "<f8", 3), ("length", "<f8"),
                           ("radius", "<f8")])
GPU_SEGMENT_DTYPE = np.dtype([("midpoint", "<f8", 3), ("direction", "<f8", 3), ("length", "<f8")])
RP_RESULT_DTYPE = np.dtype([("u_theta", "<f8"), ("u_phi", "<f8"), ("gain_total_dbi", "<f8"),
                            ("gain_theta_dbi", "<f8"), ("gain_phi_dbi", "<f8"), ("axial_ratio", "<f8"),
                            ("theta_deg", "<f8"), ("phi_deg", "<f8")])
JUNCTION_DTYPE = np.dtype([("seg_a", "<u8"), ("seg_b", "<u8"), ("sign", "<f8")])
WIRE_DTYPE = np.dtype([("tag", "<u4"), ("segments", "<u4"), ("start", "<f8", 3), ("end", "<f8", 3),
                       ("radius", "<f8")])
SOURCE_DTYPE = np.dtype([("tag", "<u4"), ("segment", "<u4"), ("v_re", "<f8"), ("v_im", "<f8")])
# LD card (fnec_load): type, tag, first and last segment, F1..F3
LOAD_DTYPE = np.dtype([("load_type", "<i4"), ("tag", "<u4"), ("seg_first", "<u4"), ("seg_last", "<u4"),
                       ("f1", "<f8"), ("f2", "<f8"), ("f3", "<f8")])
# TL card (fnec_tl) and NT card with its ten fields parsed (fnec_nt)
TL_DTYPE = np.dtype([("tag1", "<u4"), ("seg1", "<u4"), ("tag2", "<u4"), ("seg2", "<u4"), ("num_segments", "<u4"),
                     ("tl_type", "<u4"), ("z0", "<f8"), ("length", "<f8"), ("f3", "<f8")])
NT_DTYPE = np.dtype([("tag1", "<u4"), ("seg1", "<u4"), ("tag2", "<u4"), ("seg2", "<u4"), ("y11_re", "<f8"),
                     ("y11_im", "<f8"), ("y12_re", "<f8"), ("y12_im", "<f8"), ("y22_re", "<f8"), ("y22_im", "<f8")])
FEED_COLUMNS = ("seg", "v_re", "v_im", "i_re", "i_im", "z_re", "z_im")
PATTERN_COLUMNS = ("gain_total_dbi", "gain_theta_dbi", "gain_phi_dbi", "axial_ratio", "u_theta", "u_phi")

_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_U32 = ctypes.c_uint32
_I32 = ctypes.c_int32
_D = ctypes.c_double


class AccelError(RuntimeError):
    """A failed device call; ``code`` is the library status (FNEC_ERR_*)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"fnec_cuda error {code}: {msg}")
        self.code = code


class _RpCard(ctypes.Structure):
    _fields_ = [("n_theta", _U32), ("n_phi", _U32), ("theta0", _D), ("phi0", _D), ("d_theta", _D),
                ("d_phi", _D)]


class _PlaneWave(ctypes.Structure):
    _fields_ = [("ex_type", _U32), ("n_theta", _U32), ("n_phi", _U32), ("reserved", _U32), ("theta0", _D),
                ("phi0", _D), ("eta", _D), ("d_theta", _D), ("d_phi", _D), ("axial_ratio", _D)]


class _Antenna(ctypes.Structure):
    _fields_ = [("wires", _P), ("n_wires", _U32), ("sources", _P), ("n_sources", _U32), ("ground", _I32),
                ("n_freqs", _U32), ("freqs_hz", _P), ("rp", _P), ("separate_sources", _U32), ("loads", _P),
                ("n_loads", _U32), ("tls", _P), ("n_tls", _U32), ("nts", _P), ("n_nts", _U32),
                ("plane_wave", _P), ("rp_points", _P), ("n_rp_points", _U32)]


class _DeckInfo(ctypes.Structure):
    _fields_ = [("n_wires", _U32), ("n_sources", _U32), ("n_ex", _U32), ("n_loads", _U32), ("n_tls", _U32),
                ("n_nts", _U32), ("n_freqs", _U32), ("n_rp_cards", _U32), ("n_points", _U32), ("n_ne_cards", _U32),
                ("ground", _I32), ("plane_wave", _U32), ("warnings", _U32), ("runnable", _U32),
                ("why", ctypes.c_char * 200)]


class _UnitInfo(ctypes.Structure):
    _fields_ = [("antenna", _U32), ("n", _U32), ("s", _U32), ("n_feed", _U32), ("n_points", _U32),
                ("freq_hz", _D), ("cur_off", _U64), ("feed_off", _U64), ("pat_off", _U64), ("rhs", _U32),
                ("system", _U32)]


class _BatchInfo(ctypes.Structure):
    _fields_ = [("n_units", _U32), ("max_s", _U32), ("total_currents", _U64), ("total_feeds", _U64),
                ("total_points", _U64), ("device_bytes", _U64), ("h2d_bytes", _U64),
                ("kernel_launches", _U64), ("n_systems", _U32),
                ("create_ms", _D), ("antennas_ms", _D), ("alloc_ms", _D), ("alloc_device_ms", _D),
                ("alloc_pinned_ms", _D), ("alloc_mixed_ms", _D)]


class _ServerConfig(ctypes.Structure):
    _fields_ = [("precision", _I32), ("lanes", _I32), ("hbm_budget_bytes", _U64), ("max_batch", _U32),
                ("queue_cap", _U32)]


class _RequestOut(ctypes.Structure):
    _fields_ = [("currents", _P), ("feeds", _P), ("pattern", _P), ("status", _P)]


class _RequestInfo(ctypes.Structure):
    _fields_ = [("n_segments", _U32), ("n_rhs", _U32), ("n_solves", _U32), ("n_feed_rows", _U32),
                ("n_points", _U32), ("pad", _U32), ("device_bytes", _U64)]


class _RequestResult(ctypes.Structure):
    _fields_ = [("currents", _P), ("cur_stride", _U64), ("feeds", _P), ("pattern", _P), ("status", _P),
                ("n_solves", _U32), ("n_segments", _U32), ("n_feed_rows", _U32), ("n_points", _U32)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("submitted", _U64), ("completed", _U64), ("failed", _U64), ("solves", _U64), ("batches", _U64),
                ("queued", _U64), ("in_flight_bytes", _U64), ("peak_in_flight_bytes", _U64), ("max_batch", _U64),
                ("kernel_launches", _U64), ("h2d_bytes", _U64), ("d2h_bytes", _U64),
                ("plan_ms", _D), ("launch_ms", _D), ("collect_ms", _D), ("alloc_ms", _D),
                ("alloc_device_ms", _D), ("alloc_upload_ms", _D), ("alloc_pinned_ms", _D), ("alloc_mixed_ms", _D),
                ("p50_ms", _D), ("p99_ms", _D), ("mean_ms", _D), ("max_ms", _D)]


# name -> (restype, argtypes); every function declared in include/fnec_cuda.h
SIGNATURES = {
    "fnec_ctx_create": (ctypes.c_int, [ctypes.c_int, _P]),
    "fnec_ctx_destroy": (ctypes.c_int, [_P]),
    "fnec_ctx_last_error": (ctypes.c_char_p, [_P]),
    "fnec_ctx_stream": (_P, [_P]),
    "fnec_fill_zmatrix": (ctypes.c_int, [_P, _P, _U64, _D, _I32, _P]),
    "fnec_solve_hallen_resident": (ctypes.c_int, [_P, _P, _U64, _P, _P, _P, _U64, _P, _U64, _D, _I32, _I32,
                                                  _P, _P]),
    "fnec_solve_hallen": (ctypes.c_int, [_P, _P, _U64, _P, _P, _P, _U64, _P, _U64, _I32, _P, _P]),
    "fnec_rp_farfield_batch": (ctypes.c_int, [_P, _P, _U64, _P, _D, _D, _P, _U64, _P]),
    "fnec_radiation_pattern": (ctypes.c_int, [_P, _P, _U64, _P, _D, _I32, _P, _U64, _P, _P]),
    "fnec_integrate_radiated_power": (ctypes.c_int, [_P, _P, _U64, _P, _D, _I32, _P]),
    "fnec_build_geometry": (ctypes.c_int, [_P, _U32, _P, _U64, _P]),
    "fnec_abi_struct_sizes": (_U32, [_P, _U32]),
    "fnec_deck_parse": (ctypes.c_int, [ctypes.c_char_p, _P, ctypes.c_char_p, _U64]),
    "fnec_deck_destroy": (ctypes.c_int, [_P]),
    "fnec_deck_get_info": (ctypes.c_int, [_P, _P]),
    "fnec_deck_get_antenna": (ctypes.c_int, [_P, _P, _P]),
    "fnec_deck_solve": (ctypes.c_int, [_P, _P, _I32, _P, _P]),
    "fnec_near_field": (ctypes.c_int, [_P, _P, _U64, _P, _D, _P, _U64, _P, _P]),
    "fnec_microbench_zmatrix_dispatch": (ctypes.c_int, [ctypes.c_int, _U64, _U32, _P, _P, _P]),
    "fnec_enumerate_devices": (ctypes.c_int, [_P, ctypes.c_int, ctypes.c_char_p, _U64]),
    "fnec_dispatch_frequency_point": (ctypes.c_int, [ctypes.c_int, _D]),
    "fnec_measure_fp64_peak": (ctypes.c_int, [ctypes.c_int, _P, _P]),
    "fnec_measure_fp32_peak": (ctypes.c_int, [ctypes.c_int, _P]),
    "fnec_host_alloc": (ctypes.c_int, [ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]),
    "fnec_server_create": (ctypes.c_int, [_P, _P, _P]),
    "fnec_server_destroy": (ctypes.c_int, [_P]),
    "fnec_request_shape": (ctypes.c_int, [_P, _P, _I32, _P]),
    "fnec_server_submit": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "fnec_server_result": (ctypes.c_int, [_P, _U64, _P]),
    "fnec_server_next_done": (ctypes.c_int, [_P, _D, _P]),
    "fnec_server_release": (ctypes.c_int, [_P, _U64]),
    "fnec_server_poll": (ctypes.c_int, [_P, _U64, _P, _P]),
    "fnec_server_wait": (ctypes.c_int, [_P, _U64, _D, _P, _P]),
    "fnec_server_stats": (ctypes.c_int, [_P, _P, _I32]),
    "fnec_server_last_error": (ctypes.c_char_p, [_P]),
    "fnec_host_free": (ctypes.c_int, [_P]),
    "fnec_selftest_tf32x3_gemm": (ctypes.c_int, [ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64,
                                                 _P, _P, _P]),
    "fnec_radiation_pattern_noalloc": (ctypes.c_int, [_P, _U64, _P, _D, _I32, _P, _U64, _P, _P, _P]),
    "fnec_selftest_wait_timeout": (ctypes.c_int, [_I32, _I32, _U64, _P, _P]),
    "fnec_batch_set_sources": (ctypes.c_int, [_P, _U32, _P, _U32]),
    "fnec_batch_resolve": (ctypes.c_int, [_P]),
    "fnec_test_fail_device_allocation": (ctypes.c_int, [_I32]),
    "fnec_test_fill_sincospi": (ctypes.c_int, [_P, _U64, _P, _P]),
    "fnec_test_fill_rsqrt": (ctypes.c_int, [_P, _U64, _P]),
    "fnec_host_cache_release": (ctypes.c_int, [_P]),
    "fnec_device_cache_release": (ctypes.c_int, [_P, _P]),
    "fnec_batch_create": (ctypes.c_int, [_P, _P, _U32, _I32, _P]),
    "fnec_batch_destroy": (ctypes.c_int, [_P]),
    "fnec_batch_get_info": (ctypes.c_int, [_P, _P]),
    "fnec_batch_get_unit_info": (ctypes.c_int, [_P, _U32, _P]),
    "fnec_batch_upload": (ctypes.c_int, [_P]),
    "fnec_batch_run": (ctypes.c_int, [_P]),
    "fnec_batch_sync": (ctypes.c_int, [_P]),
    "fnec_batch_read": (ctypes.c_int, [_P, _P, _P, _P, _P, _P]),
    "fnec_batch_set_profiling": (ctypes.c_int, [_P, ctypes.c_int]),
    "fnec_batch_phase_ms": (ctypes.c_int, [_P, _P]),
    "fnec_batch_read_unit": (ctypes.c_int, [_P, _U32, _P, _P]),
    "fnec_batch_read_receive": (ctypes.c_int, [_P, _P]),
    "fnec_batch_read_report": (ctypes.c_int, [_P, _P, _P, _P, _P]),
    "fnec_batch_run_report": (ctypes.c_int, [_P, _P]),
    "fnec_batch_read_z": (ctypes.c_int, [_P, _U32, _P]),
    "fnec_batch_read_refinement": (ctypes.c_int, [_P, _P, _P]),
    "fnec_batch_get_schedule": (ctypes.c_int, [_P, _P]),
    "fnec_batch_set_schedule": (ctypes.c_int, [_P, _P]),
    "fnec_batch_graph_state": (ctypes.c_int, [_P, _P, _P]),
    "fnec_batch_tune": (ctypes.c_int, [_P, _U32, _P]),
    "fnec_tune_cache_save": (ctypes.c_int, [ctypes.c_char_p]),
    "fnec_tune_cache_load": (ctypes.c_int, [ctypes.c_char_p]),
    "fnec_tune_cache_clear": (ctypes.c_int, []),
    "fnec_tune_cache_size": (ctypes.c_int, [_P]),
}

_lib = None
# Live handles, released in a fixed order at interpreter exit (batches before
# the contexts they were created on): module teardown order is otherwise
# arbitrary and a batch must never outlive its context.
_live_batches = weakref.WeakSet()
_live_servers = weakref.WeakSet()
_live_contexts = weakref.WeakSet()
_shutting_down = False


@atexit.register
def _release_all():
    global _shutting_down
    for v in list(_live_servers):
        v.close()
    for b in list(_live_batches):
        b.close()
    for c in list(_live_contexts):
        c.close()
    _shutting_down = True


def lib():
    """Load libfnec_cuda.so (built in-tree by __graft_entry__.build()).

    Raises AccelError if the library is missing: the product path never
    falls back to a CPU implementation."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AccelError(ERR_NO_DEVICE, f"{LIB_PATH} is not built")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


class Context:
    """One device context (CUDA device + stream) of the library."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().fnec_ctx_create(device, ctypes.byref(h))
        if st != OK:
            raise AccelError(st, f"fnec_ctx_create(device={device})")
        self._h = h
        _live_contexts.add(self)

    @property
    def handle(self):
        return self._h

    def check(self, st: int, what: str):
        if st != OK:
            msg = lib().fnec_ctx_last_error(self._h)
            raise AccelError(st, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            for v in list(_live_servers):
                if v.ctx is self:
                    v.close()
            for b in list(_live_batches):
                if b.ctx is self:
                    b.close()
            lib().fnec_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        if _shutting_down:
            return
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def zsegments_from(segs) -> np.ndarray:
    """ZSegmentInput records from any array with mid/dir/length/radius fields."""
    out = np.zeros(len(segs), dtype=ZSEGMENT_DTYPE)
    names = segs.dtype.names
    out["midpoint"] = segs["mid"] if "mid" in names else segs["midpoint"]
    out["direction"] = segs["dir"] if "dir" in names else segs["direction"]
    out["length"] = segs["length"]
    out["radius"] = segs["radius"]
    return out


def gpu_segments_from(segs) -> np.ndarray:
    out = np.zeros(len(segs), dtype=GPU_SEGMENT_DTYPE)
    names = segs.dtype.names
    out["midpoint"] = segs["mid"] if "mid" in names else segs["midpoint"]
    out["direction"] = segs["dir"] if "dir" in names else segs["direction"]
    out["length"] = segs["length"]
    return out


# --------------------------------------------------------------------------
# reference nec_accel entry points
# --------------------------------------------------------------------------
def build_geometry(wires) -> np.ndarray:
    """build_geometry (geometry.rs:676-754) on the host: ZSEGMENT_DTYPE records
    of the GW cards' segments in card order."""
    w = np.ascontiguousarray(wires, dtype=WIRE_DTYPE)
    n = ctypes.c_uint64(0)
    st = lib().fnec_build_geometry(_ptr(w), len(w), None, 0, ctypes.byref(n))
    if st != OK:
        raise AccelError(st, "build_geometry: invalid GW card")
    out = np.zeros(n.value, dtype=ZSEGMENT_DTYPE)
    lib().fnec_build_geometry(_ptr(w), len(w), _ptr(out), n.value, ctypes.byref(n))
    return out


class Deck:
    """A NEC deck read by the library (nec_parser::parse): its cards as one
    antenna, and fnec_deck_solve's per-frequency report contract v1 text."""

    def __init__(self, text: str):
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        st = lib().fnec_deck_parse(text.encode(), ctypes.byref(h), err, len(err))
        if st != OK:
            raise AccelError(st, f"deck_parse: {err.value.decode()}")
        self._h = h

    def info(self) -> dict:
        i = _DeckInfo()
        lib().fnec_deck_get_info(self._h, ctypes.byref(i))
        d = {k: getattr(i, k) for k, _ in _DeckInfo._fields_}
        d["why"] = i.why.decode()
        return d

    def antenna(self):
        """(the C fnec_antenna view, the FR frequencies in Hz)."""
        a = _Antenna()
        n = self.info()["n_freqs"]
        f = np.zeros(max(n, 1), np.float64)
        lib().fnec_deck_get_antenna(self._h, ctypes.byref(a), _ptr(f))
        return a, f[:n]

    def solve(self, precision: int = PRECISION_FP64, ctx: Optional[Context] = None) -> str:
        ctx = ctx or default_context()
        p = ctypes.c_char_p()
        n = ctypes.c_uint64(0)
        ctx.check(lib().fnec_deck_solve(ctx.handle, self._h, int(precision), ctypes.byref(p), ctypes.byref(n)),
                  "deck_solve")
        return ctypes.string_at(p, n.value).decode()

    def close(self):
        if getattr(self, "_h", None):
            lib().fnec_deck_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fill_zmatrix(segments, freq_hz: float, ground: int = GROUND_FREE, ctx: Optional[Context] = None):
    """fill_zmatrix_wgpu (wgpu_device.rs:832): the N x N Hallen matrix,
    complex128, row-major; FP64 and with the PEC image when ground == 1."""
    ctx = ctx or default_context()
    segs = np.ascontiguousarray(segments, dtype=ZSEGMENT_DTYPE)
    n = len(segs)
    z = np.zeros((n, n), np.complex128)
    ctx.check(lib().fnec_fill_zmatrix(ctx.handle, _ptr(segs), n, float(freq_hz), int(ground), _ptr(z)),
              "fill_zmatrix")
    return z


def solve_hallen_gpu_resident(segments, rhs, cos_vec, wire_endpoints, junctions, freq_hz: float,
                              ground: int = GROUND_FREE, precision: int = PRECISION_FP64,
                              ctx: Optional[Context] = None, return_pivots: bool = False):
    """solve_hallen_gpu_resident (wgpu_device.rs:1294-1301): fill, normal
    equations and elimination on the device; returns x = [I_0..I_{N-1},
    C_0..C_{W-1}] (and the pivot rows when ``return_pivots``)."""
    ctx = ctx or default_context()
    segs = np.ascontiguousarray(segments, dtype=ZSEGMENT_DTYPE)
    n = len(segs)
    rhs = np.ascontiguousarray(rhs, np.complex128)
    cosv = np.ascontiguousarray(cos_vec, np.float64)
    ep = np.ascontiguousarray(np.asarray(wire_endpoints, dtype=np.uint64).reshape(-1, 2))
    jn = np.zeros(len(junctions), dtype=JUNCTION_DTYPE)
    for i, (a, b, s) in enumerate(junctions):
        jn[i] = (a, b, s)
    w = max(len(ep), 1)
    x = np.zeros(n + w, np.complex128)
    piv = np.zeros(n + w, np.int32)
    ctx.check(lib().fnec_solve_hallen_resident(ctx.handle, _ptr(segs), n, _ptr(rhs), _ptr(cosv), _ptr(ep),
                                               len(ep), _ptr(jn), len(jn), float(freq_hz), int(ground),
                                               int(precision), _ptr(x), _ptr(piv)),
              "solve_hallen_gpu_resident")
    return (x, piv) if return_pivots else x


def solve_hallen(z, rhs, cos_vec, wire_endpoints, junctions, precision: int = PRECISION_FP64,
                 ctx: Optional[Context] = None, return_pivots: bool = False):
    """nec_solver::solve_hallen (linear.rs:672-797) on a given Z matrix."""
    ctx = ctx or default_context()
    z = np.ascontiguousarray(z, np.complex128)
    n = z.shape[0]
    rhs = np.ascontiguousarray(rhs, np.complex128)
    cosv = np.ascontiguousarray(cos_vec, np.float64)
    ep = np.ascontiguousarray(np.asarray(wire_endpoints, dtype=np.uint64).reshape(-1, 2))
    jn = np.zeros(len(junctions), dtype=JUNCTION_DTYPE)
    for i, (a, b, s) in enumerate(junctions):
        jn[i] = (a, b, s)
    w = max(len(ep), 1)
    x = np.zeros(n + w, np.complex128)
    piv = np.zeros(n + w, np.int32)
    ctx.check(lib().fnec_solve_hallen(ctx.handle, _ptr(z), n, _ptr(rhs), _ptr(cosv), _ptr(ep), len(ep),
                                      _ptr(jn), len(jn), int(precision), _ptr(x), _ptr(piv)), "solve_hallen")
    return (x, piv) if return_pivots else x


def run_rp_farfield_batch(segments, currents, k: float, total_radiated: float, points,
                          ctx: Optional[Context] = None) -> np.ndarray:
    """run_rp_farfield_batch_wgpu (wgpu_device.rs:461-467): RpGpuResult per
    (theta, phi) point, normalised by the caller's ``total_radiated``."""
    ctx = ctx or default_context()
    segs = np.ascontiguousarray(segments, dtype=GPU_SEGMENT_DTYPE)
    cur = np.ascontiguousarray(currents, np.complex128)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 2)
    out = np.zeros(len(pts), dtype=RP_RESULT_DTYPE)
    ctx.check(lib().fnec_rp_farfield_batch(ctx.handle, _ptr(segs), len(segs), _ptr(cur), float(k),
                                           float(total_radiated), _ptr(pts), len(pts), _ptr(out)),
              "run_rp_farfield_batch")
    return out


def compute_radiation_pattern(segments, currents, freq_hz: float, points, ground: int = GROUND_FREE,
                              ctx: Optional[Context] = None):
    """compute_radiation_pattern (farfield.rs:563-647) with the power
    integral on the device.  Returns ((p, 4) gains/axial ratio, total)."""
    ctx = ctx or default_context()
    segs = np.ascontiguousarray(segments, dtype=GPU_SEGMENT_DTYPE)
    cur = np.ascontiguousarray(currents, np.complex128)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 2)
    out = np.zeros((len(pts), 4), np.float64)
    tot = np.zeros(1, np.float64)
    ctx.check(lib().fnec_radiation_pattern(ctx.handle, _ptr(segs), len(segs), _ptr(cur), float(freq_hz),
                                           int(ground), _ptr(pts), len(pts), _ptr(out), _ptr(tot)),
              "compute_radiation_pattern")
    return out, float(tot[0])


def radiation_pattern_noalloc(d_segments: int, n: int, d_currents: int, freq_hz: float, ground: int,
                              d_points: int, p: int, d_out: int, d_total: int = 0, stream: int = 0) -> int:
    """The pattern on caller-owned DEVICE buffers with no device allocation
    (for callers that cannot call cudaMalloc); returns the library status.
    Pointers are integer device addresses; the caller synchronises."""
    return lib().fnec_radiation_pattern_noalloc(d_segments, n, d_currents, float(freq_hz), int(ground),
                                                d_points, p, d_out, d_total or None, stream or None)


def integrate_radiated_power(segments, currents, freq_hz: float, pec_ground: bool,
                             ctx: Optional[Context] = None) -> float:
    """integrate_radiated_power (farfield.rs:409-417)."""
    ctx = ctx or default_context()
    segs = np.ascontiguousarray(segments, dtype=GPU_SEGMENT_DTYPE)
    cur = np.ascontiguousarray(currents, np.complex128)
    tot = np.zeros(1, np.float64)
    ctx.check(lib().fnec_integrate_radiated_power(ctx.handle, _ptr(segs), len(segs), _ptr(cur), float(freq_hz),
                                                  int(bool(pec_ground)), _ptr(tot)),
              "integrate_radiated_power")
    return float(tot[0])


def near_field(segments, currents, freq_hz: float, points, electric: bool = True, magnetic: bool = True,
               ctx: Optional[Context] = None):
    """near_e_field / near_h_field (farfield.rs:154-261): the fields of the
    segment currents at (p, 3) points in metres.  Returns (E, H), each (p, 3)
    complex, or None for the one not asked for."""
    if not (electric or magnetic):
        raise ValueError("near_field: ask for E, H or both")
    ctx = ctx or default_context()
    segs = np.ascontiguousarray(segments, dtype=GPU_SEGMENT_DTYPE)
    cur = np.ascontiguousarray(currents, np.complex128)
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    e = np.zeros((len(pts), 3), np.complex128) if electric else None
    h = np.zeros((len(pts), 3), np.complex128) if magnetic else None
    ctx.check(lib().fnec_near_field(ctx.handle, _ptr(segs), len(segs), _ptr(cur), float(freq_hz), _ptr(pts),
                                    len(pts), None if e is None else _ptr(e), None if h is None else _ptr(h)),
              "near_field")
    return e, h


@dataclass
class GpuMicrobench:
    """GpuMicrobench (wgpu_device.rs:1064-1075)."""

    n_segments: int
    n_dispatches: int
    device_init_us: int
    dispatch_min_us: int
    dispatch_median_us: int


def microbench_zmatrix_dispatch(n_segments: int, n_dispatches: int, device: int = 0) -> GpuMicrobench:
    """microbench_zmatrix_dispatch (wgpu_device.rs:1087)."""
    a, b, c = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
    st = lib().fnec_microbench_zmatrix_dispatch(device, n_segments, n_dispatches, ctypes.byref(a),
                                                ctypes.byref(b), ctypes.byref(c))
    if st != OK:
        raise AccelError(st, "microbench_zmatrix_dispatch")
    return GpuMicrobench(n_segments, n_dispatches, a.value, b.value, c.value)


def enumerate_compute_adapters() -> list:
    """enumerate_compute_adapters (wgpu_device.rs:24): CUDA device names."""
    cnt = ctypes.c_int()
    lib().fnec_enumerate_devices(ctypes.byref(cnt), -1, None, 0)
    out = []
    for i in range(cnt.value):
        buf = ctypes.create_string_buffer(256)
        lib().fnec_enumerate_devices(ctypes.byref(cnt), i, buf, 256)
        out.append({"name": buf.value.decode(), "backend": "cuda", "device_type": "DiscreteGpu"})
    return out


def selftest_tf32x3_gemm(a: np.ndarray, b: np.ndarray, device: int = 0) -> np.ndarray:
    """C = A B^T through the 3xTF32 tensor-core GEMM (A: m x k, B: n x k, FP32)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    m, k = a.shape
    n, k2 = b.shape
    if k != k2:
        raise ValueError("inner dimensions differ")
    c = np.empty((m, n), np.float32)
    st = lib().fnec_selftest_tf32x3_gemm(device, m, n, k, _ptr(a), _ptr(b), _ptr(c))
    if st != 0:
        raise AccelError(st, "selftest_tf32x3_gemm")
    return c


WAIT_GRID_ABSENT_CTA, WAIT_GRID_ALL_ARRIVE, WAIT_GEMM_LOADS_STOPPED = 0, 1, 2


def selftest_wait_timeout(which: int, wait_ns: int = 1_000_000, device: int = 0):
    """Make one bounded device wait run out on purpose (fnec_selftest_wait_timeout):
    returns (the status word the kernel left, the launch's milliseconds)."""
    st = ctypes.c_int32()
    ms = ctypes.c_double()
    rc = lib().fnec_selftest_wait_timeout(int(device), int(which), int(wait_ns), ctypes.byref(st), ctypes.byref(ms))
    if rc != OK:
        raise AccelError(rc, f"selftest_wait_timeout({which})")
    return int(st.value), float(ms.value)


def test_fail_device_allocation(after: int):
    """Test hook: the after-th batch device allocation from now on fails
    with OUT_OF_MEMORY (once); -1 disarms."""
    rc = lib().fnec_test_fail_device_allocation(int(after))
    if rc != OK:
        raise AccelError(rc, "test_fail_device_allocation")


def host_cache_release() -> int:
    """Free the page-locked host blocks the library keeps for reuse; returns
    their bytes."""
    n = ctypes.c_uint64()
    lib().fnec_host_cache_release(ctypes.byref(n))
    return int(n.value)


def device_cache_release(ctx: Optional["Context"] = None) -> int:
    """Return the device memory that destroyed batches left in the device's
    stream-ordered pool to the driver; returns its bytes."""
    c = ctx or default_context()
    n = ctypes.c_uint64()
    c.check(lib().fnec_device_cache_release(c.handle, ctypes.byref(n)), "device_cache_release")
    return int(n.value)


def test_fill_sincospi(x):
    """Test hook: the mixed fill's own sin(pi x), cos(pi x), run on the host
    (0 <= x < 2^50)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    s, c = np.empty_like(x), np.empty_like(x)
    rc = lib().fnec_test_fill_sincospi(_ptr(x), len(x), _ptr(s), _ptr(c))
    if rc != OK:
        raise AccelError(rc, "test_fill_sincospi")
    return s, c


def test_fill_rsqrt(x):
    """Test hook: the mixed fill's reciprocal square root, run on the
    current device (normal, finite, positive x; at most 2^20 values)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty_like(x)
    rc = lib().fnec_test_fill_rsqrt(_ptr(x), len(x), _ptr(out))
    if rc != OK:
        raise AccelError(rc, "test_fill_rsqrt")
    return out


def measure_fp32_peak(device: int = 0) -> float:
    """FP32 FFMA throughput of the GPU in TFLOP/s."""
    a = ctypes.c_double()
    st = lib().fnec_measure_fp32_peak(device, ctypes.byref(a))
    if st != 0:
        raise AccelError(st, "measure_fp32_peak")
    return a.value


def measure_fp64_peak(device: int = 0):
    """(fused DFMA, separately rounded DMUL+DADD) TFLOP/s of this GPU."""
    a, b = ctypes.c_double(), ctypes.c_double()
    st = lib().fnec_measure_fp64_peak(device, ctypes.byref(a), ctypes.byref(b))
    if st != OK:
        raise AccelError(st, "measure_fp64_peak")
    return a.value, b.value


HYBRID_GPU_CANDIDATE = 0
GPU_ONLY = 1


def dispatch_frequency_point(request_kind: int, freq_hz: float) -> str:
    """dispatch_frequency_point (lib.rs:92): "RunOnGpu" when a device exists."""
    return "RunOnGpu" if lib().fnec_dispatch_frequency_point(int(request_kind), float(freq_hz)) == 1 \
        else "NoDevice"


# --------------------------------------------------------------------------
# batched pipeline
# --------------------------------------------------------------------------
@dataclass
class Antenna:
    """One geometry: GW wires, voltage EX sources, ground, FR frequencies, an
    optional RP card (n_theta, n_phi, theta0, phi0, d_theta, d_phi),
    optional LD, TL and NT cards (LOAD_DTYPE / TL_DTYPE / NT_DTYPE arrays,
    deck order) and an optional plane-wave EX card (plane_wave(...); the
    sources must then be empty)."""

    wires: np.ndarray
    sources: np.ndarray
    freqs_hz: Sequence[float]
    ground: int = GROUND_FREE
    rp: Optional[tuple] = None
    separate_sources: bool = False  # each source its own right-hand side on one factorisation
    loads: Optional[np.ndarray] = None
    tls: Optional[np.ndarray] = None
    nts: Optional[np.ndarray] = None
    plane_wave: Optional[tuple] = None
    rp_points: Optional[np.ndarray] = None  # (p, 2) theta, phi degrees: several RP cards' points (rp None)


def plane_wave(ex_type=1, theta0=0.0, phi0=0.0, eta=0.0, n_theta=1, n_phi=1, d_theta=0.0, d_phi=0.0,
               axial_ratio=0.0) -> tuple:
    """A plane-wave EX card (type 1 linear, 2 right / 3 left elliptic): I2 =
    n_theta, I3 = n_phi, F1..F6 = theta0, phi0, eta, d_theta, d_phi, axial
    ratio.  Its directions are the receive sweep (theta outer, phi inner)."""
    return (int(ex_type), int(n_theta), int(n_phi), float(theta0), float(phi0), float(eta), float(d_theta),
            float(d_phi), float(axial_ratio))


def wires_array(wires) -> np.ndarray:
    """wires: iterable of (tag, segments, start3, end3, radius)."""
    arr = np.zeros(len(wires), dtype=WIRE_DTYPE)
    for i, (tag, nseg, s, e, r) in enumerate(wires):
        arr[i] = (tag, nseg, s, e, r)
    return arr


def loads_array(loads) -> np.ndarray:
    """loads: iterable of LD cards (type, tag, seg_first, seg_last, f1, f2, f3)."""
    arr = np.zeros(len(loads), dtype=LOAD_DTYPE)
    for i, (t, tag, s0, s1, f1, f2, f3) in enumerate(loads):
        arr[i] = (t, tag, s0, s1, f1, f2, f3)
    return arr


def tls_array(tls) -> np.ndarray:
    """tls: iterable of TL cards (tag1, seg1, tag2, seg2, num_segments, tl_type, z0, length, f3)."""
    arr = np.zeros(len(tls), dtype=TL_DTYPE)
    for i, t in enumerate(tls):
        arr[i] = tuple(t)
    return arr


def nts_array(nts) -> np.ndarray:
    """nts: iterable of NT cards (tag1, seg1, tag2, seg2, y11_re, y11_im, y12_re, y12_im, y22_re, y22_im)."""
    arr = np.zeros(len(nts), dtype=NT_DTYPE)
    for i, t in enumerate(nts):
        arr[i] = tuple(t)
    return arr


def sources_array(sources) -> np.ndarray:
    """sources: iterable of (tag, segment, complex voltage)."""
    arr = np.zeros(len(sources), dtype=SOURCE_DTYPE)
    for i, (tag, seg, v) in enumerate(sources):
        arr[i] = (tag, seg, complex(v).real, complex(v).imag)
    return arr


@dataclass
class BatchResult:
    currents: list                 # per unit: complex128[N]
    feeds: list                    # per unit: (n_feed, 7) array
    pattern: list                  # per unit: (n_points, 6) array
    status: np.ndarray             # per unit int32
    total_radiated: np.ndarray
    units: list = field(default_factory=list)


def _antenna_struct(a, keep: list):
    """The C fnec_antenna of an Antenna; the arrays it points to go to keep."""
    w = np.ascontiguousarray(a.wires, dtype=WIRE_DTYPE)
    s = np.ascontiguousarray(a.sources, dtype=SOURCE_DTYPE)
    f = np.ascontiguousarray(np.asarray(a.freqs_hz, np.float64))
    rp = None
    if a.rp is not None:
        rp = _RpCard(*[int(a.rp[0]), int(a.rp[1])] + [float(v) for v in a.rp[2:6]])
    def opt(x, dt):
        return None if x is None or len(x) == 0 else np.ascontiguousarray(x, dtype=dt)

    ld, tl, nt = opt(a.loads, LOAD_DTYPE), opt(a.tls, TL_DTYPE), opt(a.nts, NT_DTYPE)
    pw = None
    if a.plane_wave is not None:
        t, nth, nph, th0, ph0, eta, dth, dph, ar = a.plane_wave
        pw = _PlaneWave(t, nth, nph, 0, th0, ph0, eta, dth, dph, ar)
    rpp = None if a.rp_points is None else np.ascontiguousarray(a.rp_points, np.float64).reshape(-1, 2)
    keep += [w, s, f, rp, ld, tl, nt, pw, rpp]
    return _Antenna(_ptr(w), len(w), _ptr(s), len(s), int(a.ground), len(f), _ptr(f),
                    ctypes.cast(ctypes.pointer(rp), _P) if rp is not None else None,
                    int(bool(a.separate_sources)), _ptr(ld), 0 if ld is None else len(ld),
                    _ptr(tl), 0 if tl is None else len(tl), _ptr(nt), 0 if nt is None else len(nt),
                    ctypes.cast(ctypes.pointer(pw), _P) if pw is not None else None, _ptr(rpp),
                    0 if rpp is None else len(rpp))


class _Schedule(ctypes.Structure):
    _fields_ = [("grid_panels", ctypes.c_int32), ("class_shift", ctypes.c_int32), ("gram_tensor", ctypes.c_int32),
                ("gmres_cluster", ctypes.c_int32), ("grid_gmres", ctypes.c_int32), ("graph", ctypes.c_int32),
                ("factor_streams", ctypes.c_int32), ("unit_factor", ctypes.c_int32),
                ("block_inverse", ctypes.c_int32), ("tensor_trailing", ctypes.c_int32),
                ("gmres_ctas_per_sm", ctypes.c_int32), ("factor_pivoting", ctypes.c_int32)]


class _TuneReport(ctypes.Structure):
    _fields_ = [("best", _Schedule), ("default_ms", ctypes.c_double), ("best_ms", ctypes.c_double),
                ("candidates", ctypes.c_uint32), ("from_cache", ctypes.c_uint32), ("key", ctypes.c_char * 96)]


GRAPH_NONE, GRAPH_READY, GRAPH_FAILED = 0, 1, -1


def _sched_dict(s: _Schedule) -> dict:
    return {k: int(getattr(s, k)) for k, _ in _Schedule._fields_}


def tune_cache_save(path: str):
    """Write the process-wide tuning cache (shape key -> schedule) as text."""
    if lib().fnec_tune_cache_save(str(path).encode()) != OK:
        raise AccelError(ERR_BAD_ARG, f"tune_cache_save: cannot write {path}")


def tune_cache_load(path: str):
    """Merge a saved tuning cache; a malformed file changes nothing."""
    if lib().fnec_tune_cache_load(str(path).encode()) != OK:
        raise AccelError(ERR_BAD_ARG, f"tune_cache_load: cannot read {path} (missing or malformed)")


def tune_cache_clear():
    lib().fnec_tune_cache_clear()


def tune_cache_size() -> int:
    n = ctypes.c_uint32()
    lib().fnec_tune_cache_size(ctypes.byref(n))
    return int(n.value)


class HallenBatch:
    """A planned, device-resident batch of per-frequency Hallen solves."""

    def __init__(self, antennas: Sequence[Antenna], precision: int = PRECISION_FP64,
                 ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self._keep = []
        arr = (_Antenna * len(antennas))()
        for i, a in enumerate(antennas):
            arr[i] = _antenna_struct(a, self._keep)
        self._keep.append(arr)
        h = ctypes.c_void_p()
        self.ctx.check(lib().fnec_batch_create(self.ctx.handle, arr, len(antennas), int(precision),
                                               ctypes.byref(h)), "batch_create")
        self._h = h
        _live_batches.add(self)
        info = _BatchInfo()
        lib().fnec_batch_get_info(self._h, ctypes.byref(info))
        self.info = info
        self._units = None  # per-unit descriptions, read on first use
        # host result buffers, allocated once in page-locked memory: the
        # library copies straight into them
        self._host = []
        self._cur = self._pinned((max(info.total_currents, 1),), np.complex128)
        self._feed = self._pinned((max(info.total_feeds, 1), 7), np.float64)
        self._pat = self._pinned((max(info.total_points, 1), 6), np.float64)
        self._pat4 = self._pinned((max(info.total_points, 1), 4), np.float64)
        self._status = self._pinned((max(info.n_units, 1),), np.int32)
        self._total = self._pinned((max(info.n_units, 1),), np.float64)

    def upload(self):
        self.ctx.check(lib().fnec_batch_upload(self._h), "batch_upload")

    def run(self):
        self.ctx.check(lib().fnec_batch_run(self._h), "batch_run")

    def sync(self):
        self.ctx.check(lib().fnec_batch_sync(self._h), "batch_sync")

    @property
    def schedule(self) -> dict:
        """How the pipeline launches (grid_panels, class_shift, gram_tensor,
        gmres_cluster, grid_gmres, graph, factor_streams, unit_factor,
        block_inverse, tensor_trailing, gmres_ctas_per_sm, factor_pivoting)."""
        s = _Schedule()
        self.ctx.check(lib().fnec_batch_get_schedule(self._h, ctypes.byref(s)), "batch_get_schedule")
        return _sched_dict(s)

    @schedule.setter
    def schedule(self, values: dict):
        s = _Schedule()
        lib().fnec_batch_get_schedule(self._h, ctypes.byref(s))
        for k, v in values.items():
            if k not in dict(_Schedule._fields_):
                raise KeyError(k)
            setattr(s, k, int(v))
        self.ctx.check(lib().fnec_batch_set_schedule(self._h, ctypes.byref(s)), "batch_set_schedule")

    def graph_state(self):
        """(GRAPH_NONE | GRAPH_READY | GRAPH_FAILED, kernel launches per replay)."""
        st, n = ctypes.c_int32(), ctypes.c_uint64()
        self.ctx.check(lib().fnec_batch_graph_state(self._h, ctypes.byref(st), ctypes.byref(n)), "batch_graph_state")
        return int(st.value), int(n.value)

    def tune(self, reps: int = 3) -> dict:
        """Time candidate schedules on this batch, keep the fastest and cache
        it for batches of the same shape (reps=0: apply a cached one only)."""
        r = _TuneReport()
        self.ctx.check(lib().fnec_batch_tune(self._h, int(reps), ctypes.byref(r)), "batch_tune")
        return {"best": _sched_dict(r.best), "default_ms": r.default_ms, "best_ms": r.best_ms,
                "candidates": int(r.candidates), "from_cache": bool(r.from_cache), "key": r.key.decode()}

    @property
    def kernel_launches(self) -> int:
        info = _BatchInfo()
        lib().fnec_batch_get_info(self._h, ctypes.byref(info))
        return int(info.kernel_launches)

    @property
    def h2d_bytes(self) -> int:
        info = _BatchInfo()
        lib().fnec_batch_get_info(self._h, ctypes.byref(info))
        return int(info.h2d_bytes)

    def read_raw(self, currents=True, feeds=True, pattern=True):
        self.ctx.check(lib().fnec_batch_read(self._h, _ptr(self._cur) if currents else None,
                                             _ptr(self._feed) if feeds else None,
                                             _ptr(self._pat) if pattern else None, _ptr(self._status),
                                             _ptr(self._total)), "batch_read")
        return self._cur, self._feed, self._pat, self._status, self._total

    def read_report(self, pattern: bool = True):
        """The report's results (fnec_batch_read_report): currents, feeds,
        the 4 report columns of every pattern point, status; views of the
        batch's page-locked buffers.  pattern=False after run_report, which
        has streamed the columns already."""
        self.ctx.check(lib().fnec_batch_read_report(self._h, _ptr(self._cur), _ptr(self._feed),
                                                    _ptr(self._pat4) if pattern else None, _ptr(self._status)),
                       "batch_read_report")
        return self._cur, self._feed, self._pat4, self._status

    def run_report(self):
        """fnec_batch_run_report: a run whose report pattern columns are
        copied into the batch's page-locked buffer chunk by chunk behind the
        far field; read_report(pattern=False) then completes the step."""
        self.ctx.check(lib().fnec_batch_run_report(self._h, _ptr(self._pat4)), "batch_run_report")

    def d2h_report_bytes(self) -> int:
        i = self.info
        return int(4 * i.n_systems + 16 * i.total_currents + 56 * i.total_feeds + 32 * i.total_points)

    def d2h_bytes(self, currents=True, feeds=True, pattern=True) -> int:
        i = self.info
        b = 4 * i.n_systems + 8 * i.n_units
        if currents:
            b += 16 * sum(u["s"] for u in self.units)
        if feeds:
            b += 56 * i.total_feeds
        if pattern:
            b += 48 * i.total_points
        return int(b)

    def read(self, copy: bool = True) -> BatchResult:
        """Results of the last run.  copy=False returns views of the batch's
        page-locked result buffers: valid until the next read or close."""
        cur, feed, pat, st, tot = self.read_raw()
        cp = (lambda a: a.copy()) if copy else (lambda a: a)
        res = BatchResult([], [], [], cp(st[: len(self.units)]), cp(tot[: len(self.units)]), self.units)
        for u in self.units:
            res.currents.append(cp(cur[u["cur_off"]: u["cur_off"] + u["n"]]))
            res.feeds.append(cp(feed[u["feed_off"]: u["feed_off"] + u["n_feed"]]))
            res.pattern.append(cp(pat[u["pat_off"]: u["pat_off"] + u["n_points"]]))
        return res

    PHASES = ("expand", "rhs", "fill", "gram", "factor", "solve", "feed", "farfield")

    def set_profiling(self, on: bool = True):
        self.ctx.check(lib().fnec_batch_set_profiling(self._h, int(on)), "batch_set_profiling")

    def phase_ms(self) -> dict:
        ms = np.zeros(len(self.PHASES), np.float64)
        self.ctx.check(lib().fnec_batch_phase_ms(self._h, _ptr(ms)), "batch_phase_ms")
        return dict(zip(self.PHASES, ms.tolist()))

    def read_unit(self, unit: int):
        u = self.units[unit]
        x = np.zeros(u["s"], np.complex128)
        piv = np.zeros(u["s"], np.int32)
        self.ctx.check(lib().fnec_batch_read_unit(self._h, unit, _ptr(x), _ptr(piv)), "batch_read_unit")
        return x, piv

    def read_receive(self) -> np.ndarray:
        """(n_units, 3): theta, phi and the receive response in dB of every
        plane-wave unit (solve_session.rs:313-375); NaN rows for the others."""
        out = np.zeros((len(self.units), 3), np.float64)
        self.ctx.check(lib().fnec_batch_read_receive(self._h, _ptr(out)), "batch_read_receive")
        return out

    def refinement_stats(self):
        """(GMRES iterations, final preconditioned relative residual) per unit
        of the last run of a mixed-precision batch."""
        it = np.zeros(len(self.units), np.int32)
        rs = np.zeros(len(self.units), np.float64)
        self.ctx.check(lib().fnec_batch_read_refinement(self._h, _ptr(it), _ptr(rs)), "batch_read_refinement")
        return it, rs

    def read_z(self, unit: int) -> np.ndarray:
        u = self.units[unit]
        z = np.zeros((u["n"], u["n"]), np.complex128)
        self.ctx.check(lib().fnec_batch_read_z(self._h, unit, _ptr(z)), "batch_read_z")
        return z

    def solve(self) -> BatchResult:
        self.run()
        self.sync()
        return self.read()

    def set_sources(self, antenna: int, sources):
        """New voltage sources for one antenna of a batch that has run
        (fnec_batch_set_sources); sources: a SOURCE_DTYPE array or
        (tag, segment, voltage) tuples, giving every right-hand side its
        planned numbers of resolved sources and feed rows."""
        arr = sources if isinstance(sources, np.ndarray) else sources_array(sources)
        arr = np.ascontiguousarray(arr, dtype=SOURCE_DTYPE)
        self.ctx.check(lib().fnec_batch_set_sources(self._h, int(antenna), _ptr(arr) if len(arr) else None, len(arr)),
                       "batch_set_sources")

    def resolve(self, read: bool = True):
        """Solve every unit again on the resident factorisations with the
        current sources (fnec_batch_resolve); read=True waits and returns the
        results, read=False only enqueues the work on the batch's stream."""
        self.ctx.check(lib().fnec_batch_resolve(self._h), "batch_resolve")
        if not read:
            return None
        self.sync()
        return self.read()

    @property
    def units(self) -> list:
        """One dict of _UnitInfo fields per solve unit, read from the library
        on first use (one call per unit)."""
        if self._units is None:
            us = []
            for u in range(self.info.n_units):
                ui = _UnitInfo()
                lib().fnec_batch_get_unit_info(self._h, u, ctypes.byref(ui))
                us.append({k: getattr(ui, k) for k, _ in _UnitInfo._fields_})
            self._units = us
        return self._units

    def _pinned(self, shape, dtype):
        nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        p = ctypes.c_void_p()
        st = lib().fnec_host_alloc(nbytes, ctypes.byref(p))
        if st != 0:
            raise AccelError(st, "host_alloc")
        self._host.append(p)
        buf = (ctypes.c_char * nbytes).from_address(p.value)
        return np.frombuffer(buf, dtype=dtype).reshape(shape)

    def close(self):
        if getattr(self, "_h", None):
            lib().fnec_batch_destroy(self._h)
            self._h = None
        for p in getattr(self, "_host", []):
            lib().fnec_host_free(p)
        self._host = []

    def __del__(self):
        if _shutting_down:
            return
        try:
            self.close()
        except Exception:
            pass


REQ_QUEUED, REQ_RUNNING, REQ_DONE = 0, 1, 2


def _view(ptr, dtype, shape, strides=None):
    """A numpy view of library-owned host memory (no copy)."""
    dt = np.dtype(dtype)
    if strides is None:
        nbytes = int(np.prod(shape)) * dt.itemsize
    else:
        nbytes = sum((n - 1) * st for n, st in zip(shape, strides)) + dt.itemsize if all(shape) else 0
    if nbytes == 0 or not ptr:
        return np.zeros(shape, dt)
    buf = (ctypes.c_char * nbytes).from_address(ptr)
    return np.ndarray(shape, dt, buffer=buf, strides=strides)


class Request:
    """One submitted request.  With copy_out its results are copied into
    its own arrays (currents, feeds, pattern, status); otherwise they are
    read in place from the server's page-locked memory (result()) until
    release()."""

    def __init__(self, server, antenna, copy_out, currents, feeds, pattern):
        self.server = server
        self.antenna = antenna
        self.copy_out = copy_out
        self.info = _RequestInfo()
        self.want = (currents, feeds, pattern)
        self.currents = self.feeds = self.pattern = self.status = None
        self.ticket = None
        self.latency_ms = None
        self.state = REQ_QUEUED
        self._keep = []

    def _alloc(self):
        i = self.info
        c, f, p = self.want
        self.currents = np.zeros((i.n_solves, i.n_segments), np.complex128) if c else None
        self.feeds = np.zeros((max(i.n_feed_rows, 1), 7), np.float64) if f else None
        self.pattern = np.zeros((i.n_solves, i.n_points, 6), np.float64) if (p and i.n_points) else None
        self.status = np.zeros(i.n_solves, np.int32)

    @property
    def n_solves(self):
        return self.info.n_solves

    def result(self):
        """(currents, feeds, pattern, status) of a finished request; views of
        server memory (valid until release) unless submitted with copy_out."""
        if self.copy_out:
            return self.currents, self.feeds, self.pattern, self.status
        r = _RequestResult()
        st = lib().fnec_server_result(self.server._h, self.ticket, ctypes.byref(r))
        if st != 0:
            raise AccelError(st, "server_result")
        cur = _view(r.currents, np.complex128, (r.n_solves, r.n_segments), (16 * r.cur_stride, 16))
        feeds = _view(r.feeds, np.float64, (r.n_feed_rows, 7))
        pat = _view(r.pattern, np.float64, (r.n_solves, r.n_points, 6)) if r.n_points else None
        status = _view(r.status, np.int32, (r.n_solves,))
        return cur, feeds, pat, status

    def feed_z(self, solve: int = 0) -> complex:
        """Feedpoint impedance of a solve's first feed row (columns 5, 6)."""
        feeds = self.result()[1]
        rows_per = len(feeds) // max(self.n_solves, 1)
        r = feeds[solve * rows_per]
        return complex(r[5], r[6])

    def release(self):
        if self.ticket is not None and self.server._h:
            lib().fnec_server_release(self.server._h, self.ticket)
            self.server._pending.pop(self.ticket, None)
        self.ticket = None


class Server:
    """Continuous-batching solve server (fnec_server_*): submit decks as they
    arrive; lanes (each a CUDA stream with its own host thread) admit them by
    HBM budget and deliver each request's results."""

    def __init__(self, precision: int = PRECISION_MIXED, lanes: int = 2, hbm_budget_bytes: int = 32 << 30,
                 max_batch: int = 64, queue_cap: int = 0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.precision = int(precision)
        cfg = _ServerConfig(self.precision, int(lanes), int(hbm_budget_bytes), int(max_batch), int(queue_cap))
        h = ctypes.c_void_p()
        self.ctx.check(lib().fnec_server_create(self.ctx.handle, ctypes.byref(cfg), ctypes.byref(h)),
                       "server_create")
        self._h = h
        self._pending = {}
        _live_servers.add(self)

    def shape(self, antenna):
        keep = []
        a = _antenna_struct(antenna, keep)
        info = _RequestInfo()
        self.ctx.check(lib().fnec_request_shape(self.ctx.handle, ctypes.byref(a), self.precision,
                                                ctypes.byref(info)), "request_shape")
        return info

    def submit(self, antenna, copy_out: bool = False, currents: bool = True, feeds: bool = True,
               pattern: bool = True, tag=None) -> Request:
        """Queue a deck; `tag` is kept on the Request (e.g. the caller's index)."""
        keep = []
        a = _antenna_struct(antenna, keep)
        req = Request(self, antenna, copy_out, currents, feeds, pattern)
        req.tag = tag
        req._keep = keep
        out = None
        if copy_out:
            self.ctx.check(lib().fnec_request_shape(self.ctx.handle, ctypes.byref(a), self.precision,
                                                    ctypes.byref(req.info)), "request_shape")
            req._alloc()
            out = _RequestOut(_ptr(req.currents), _ptr(req.feeds), _ptr(req.pattern), _ptr(req.status))
        t = ctypes.c_uint64()
        st = lib().fnec_server_submit(self._h, ctypes.byref(a), ctypes.byref(out) if out is not None else None,
                                      ctypes.byref(t), ctypes.byref(req.info))
        if st != 0:
            raise AccelError(st, "server_submit")
        req.ticket = t.value
        self._pending[req.ticket] = req  # keeps output arrays alive until released
        return req

    def _finish(self, req, state, lat):
        req.state = state
        if state == REQ_DONE or state < 0:
            req.latency_ms = lat
        if state < 0:
            msg = lib().fnec_server_last_error(self._h)
            raise AccelError(state, f"request failed: {msg.decode() if msg else ''}")

    def poll(self, req: Request) -> bool:
        if req.state == REQ_DONE:
            return True
        state, lat = ctypes.c_int32(), ctypes.c_double()
        st = lib().fnec_server_poll(self._h, req.ticket, ctypes.byref(state), ctypes.byref(lat))
        if st != 0:
            raise AccelError(st, "server_poll")
        self._finish(req, state.value, lat.value)
        return req.state == REQ_DONE

    def wait(self, req: Request, timeout_ms: float = 120000.0) -> Request:
        if req.state == REQ_DONE:
            return req
        state, lat = ctypes.c_int32(), ctypes.c_double()
        st = lib().fnec_server_wait(self._h, req.ticket, float(timeout_ms), ctypes.byref(state), ctypes.byref(lat))
        if st != 0:
            raise AccelError(st, "server_wait")
        self._finish(req, state.value, lat.value)
        return req

    def next_done(self, timeout_ms: float = 1000.0) -> Optional[Request]:
        """The next finished request in completion order (None on timeout)."""
        t = ctypes.c_uint64()
        st = lib().fnec_server_next_done(self._h, float(timeout_ms), ctypes.byref(t))
        if st == ERR_TIMEOUT:
            return None
        if st != 0:
            raise AccelError(st, "server_next_done")
        req = self._pending.get(t.value)
        t_end = time.monotonic() + 1.0
        while req is None and time.monotonic() < t_end:  # its submit() is still returning
            time.sleep(0)
            req = self._pending.get(t.value)
        if req is not None:
            state, lat = ctypes.c_int32(), ctypes.c_double()
            lib().fnec_server_poll(self._h, req.ticket, ctypes.byref(state), ctypes.byref(lat))
            self._finish(req, state.value, lat.value)
        return req

    def stats(self, reset: bool = False) -> dict:
        s = _ServerStats()
        self.ctx.check(lib().fnec_server_stats(self._h, ctypes.byref(s), int(reset)), "server_stats")
        return {k: getattr(s, k) for k, _ in _ServerStats._fields_}

    def close(self):
        if getattr(self, "_h", None):
            lib().fnec_server_destroy(self._h)  # finishes queued and running requests
            self._h = None
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        if _shutting_down:
            return
        try:
            self.close()
        except Exception:
            pass
