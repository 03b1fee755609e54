"""CPU checks of the C ABI: the library loads without a GPU, exports every
function include/fnec_cuda.h declares, the Python mirror binds exactly that
set, and device entry points fail loudly (no CPU fallback) on a host with
no CUDA device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "fnec_cuda.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fnec_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_reference_entry_points():
    names = header_functions()
    for required in ("fnec_fill_zmatrix", "fnec_solve_hallen_resident", "fnec_solve_hallen",
                     "fnec_rp_farfield_batch", "fnec_radiation_pattern", "fnec_integrate_radiated_power",
                     "fnec_microbench_zmatrix_dispatch", "fnec_enumerate_devices",
                     "fnec_dispatch_frequency_point", "fnec_batch_create", "fnec_batch_run"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import nec_accel

    L = ctypes.CDLL(nec_accel.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(L, n)]
    assert not missing, missing


def test_python_mirror_binds_exactly_the_header():
    import nec_accel

    assert sorted(nec_accel.SIGNATURES) == header_functions()
    nec_accel.lib()


def test_no_device_is_an_error_not_a_fallback():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import nec_accel

    with pytest.raises(nec_accel.AccelError) as ei:
        nec_accel.Context(0)
    assert ei.value.code == nec_accel.ERR_NO_DEVICE
    assert nec_accel.dispatch_frequency_point(nec_accel.GPU_ONLY, 14.2e6) == "NoDevice"


def test_tune_cache_file_round_trip(tmp_path):
    """The tuning cache is host state: its text file loads, saves and
    refuses malformed input without changing the cache."""
    import nec_accel as acc

    acc.tune_cache_clear()
    good = tmp_path / "tune.txt"
    good.write_text("# shape key, then every schedule field\n"
                    "p1.sm148.ns8.nu8.smax9.smean8.gp0.gg0.tc1.cm1 grid_panels=1 class_shift=2 gram_tensor=0 "
                    "gmres_cluster=1 grid_gmres=1 graph=1 factor_streams=4 unit_factor=0 block_inverse=1 tensor_trailing=1 gmres_ctas_per_sm=4 factor_pivoting=1\n"
                    "p0.sm148.ns12.nu12.smax10.smean8.gp1.gg0.tc0.cm1 grid_panels=0 class_shift=1 gram_tensor=1 "
                    "gmres_cluster=1 grid_gmres=1 graph=0 factor_streams=1 unit_factor=1 block_inverse=0 tensor_trailing=0 gmres_ctas_per_sm=3 factor_pivoting=0\n")
    acc.tune_cache_load(good)
    assert acc.tune_cache_size() == 2
    out = tmp_path / "saved.txt"
    acc.tune_cache_save(out)
    lines = sorted(out.read_text().split("\n")[:-1])
    assert lines == sorted(l for l in good.read_text().split("\n")[1:] if l)
    bad = tmp_path / "bad.txt"
    for text in ("k grid_panels=1 class_shift=3 gram_tensor=1 gmres_cluster=1 grid_gmres=1 graph=1 factor_streams=1 unit_factor=1 block_inverse=0 tensor_trailing=0 gmres_ctas_per_sm=3 factor_pivoting=0\n",  # range
                 "k grid_panels=1 class_shift=1 gram_tensor=1 gmres_cluster=3 grid_gmres=1 graph=1 factor_streams=1 unit_factor=1 block_inverse=0 tensor_trailing=0 gmres_ctas_per_sm=3 factor_pivoting=0\n",  # cluster
                 "k grid_panels=1 class_shift=1\n",  # fields missing
                 "k grid_panels=1 class_shift=1 gram_tensor=1 gmres_cluster=1 grid_gmres=1 graph=1 factor_streams=3 unit_factor=1 block_inverse=0 tensor_trailing=0 gmres_ctas_per_sm=3 factor_pivoting=0\n",
                 "k grid_panels=1 tile=7 class_shift=1 gram_tensor=1 gmres_cluster=1 grid_gmres=1 graph=1 factor_streams=1 unit_factor=1 block_inverse=0 tensor_trailing=0 gmres_ctas_per_sm=3 factor_pivoting=0\n"):
        bad.write_text(text)
        with pytest.raises(acc.AccelError):
            acc.tune_cache_load(bad)
        assert acc.tune_cache_size() == 2
    with pytest.raises(acc.AccelError):
        acc.tune_cache_load(tmp_path / "absent.txt")
    acc.tune_cache_clear()
    assert acc.tune_cache_size() == 0


def test_struct_layouts_match_the_library():
    """Every public struct's size as compiled into the library equals its
    mirror's (numpy dtypes for the card arrays, ctypes for the rest), so a
    field added on one side only is caught without a GPU."""
    import ctypes

    import numpy as np

    import nec_accel as acc

    n = acc.lib().fnec_abi_struct_sizes(None, 0)
    sizes = (ctypes.c_uint64 * n)()
    acc.lib().fnec_abi_struct_sizes(sizes, n)
    mirror = [acc.WIRE_DTYPE.itemsize, acc.SOURCE_DTYPE.itemsize, ctypes.sizeof(acc._RpCard),
              ctypes.sizeof(acc._PlaneWave), acc.LOAD_DTYPE.itemsize, acc.TL_DTYPE.itemsize, acc.NT_DTYPE.itemsize,
              ctypes.sizeof(acc._Antenna), ctypes.sizeof(acc._UnitInfo), ctypes.sizeof(acc._BatchInfo),
              ctypes.sizeof(acc._DeckInfo), ctypes.sizeof(acc._ServerConfig), ctypes.sizeof(acc._RequestOut),
              ctypes.sizeof(acc._RequestInfo), ctypes.sizeof(acc._RequestResult), ctypes.sizeof(acc._ServerStats),
              ctypes.sizeof(acc._Schedule), ctypes.sizeof(acc._TuneReport), acc.ZSEGMENT_DTYPE.itemsize,
              acc.GPU_SEGMENT_DTYPE.itemsize, acc.RP_RESULT_DTYPE.itemsize, acc.JUNCTION_DTYPE.itemsize]
    assert list(sizes) == mirror
    assert np.dtype(acc.WIRE_DTYPE).itemsize == 64
