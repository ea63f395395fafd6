"""The C ABI library on the CPU: it loads, exports every declared symbol, and
rejects bad arguments before touching the device."""
import ctypes as C
import pathlib
import re

import numpy as np
import pytest

import mvs_b200 as M

ROOT = pathlib.Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "mvs_b200.h").read_text()
    return sorted(set(re.findall(r"\b(mvs_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) > 40
    missing = [s for s in syms if not hasattr(M.lib(), s)]
    assert not missing, missing


def test_version_and_error_string():
    assert M.lib().mvs_version() >= 10000
    assert isinstance(M.lib().mvs_last_error(), bytes)


@pytest.mark.parametrize("field,value", [("window", 4), ("window", 1), ("window", 17), ("n_views", 0),
                                         ("n_planes", 0), ("width", 0), ("moments", 7), ("mode", 5), ("width", 6)])
def test_sweep_descriptor_validation(field, value):
    d = M.sweep_desc(64, 48, 2, 16, 9)
    setattr(d, field, value)
    assert M.lib().mvs_sweep_workspace_bytes(C.byref(d)) == 0
    rc = M.lib().mvs_sweep(C.byref(d), None, None, None, None, None, None, None, None, None, 0, None)
    assert rc == M.MVS_ERR_ARG
    assert M.lib().mvs_last_error()


def test_sweep_workspace_sizes():
    d = M.sweep_desc(640, 480, 8, 256, 9)
    # per view: one winner word per pixel and view, then each source pixel's 2x2 neighbourhood
    assert M.sweep_workspace_bytes(d) == 640 * 480 * 8 * 8 + 640 * 480 * 8 * 16
    d.mode = M.SWEEP_AGGREGATED
    # one winner word per pixel, then each source pixel's 2x2 neighbourhood (16 bytes per view)
    assert M.sweep_workspace_bytes(d) == 640 * 480 * 8 + 640 * 480 * 8 * 16


def test_null_pointer_and_size_errors():
    L = M.lib()
    d = M.sweep_desc(64, 48, 2, 16, 9)
    assert L.mvs_sweep(C.byref(d), None, None, None, None, None, None, None, None, None, 0, None) == M.MVS_ERR_ARG
    h = C.c_void_p()
    assert L.mvs_fusion_create(8, 8, 8, 11, None, None, C.byref(h)) == M.MVS_ERR_ARG
    assert L.mvs_fusion_create(0, 8, 8, 7, None, None, C.byref(h)) == M.MVS_ERR_ARG
    assert L.mvs_tvl1_denoise(1, 1, None, None, 0.0, 1.0, None, None, 0, None) == M.MVS_ERR_ARG
    assert L.mvs_tgv2_run(8, 8, 0, *([None] * 7), 0, 1.0, None, None, None, None, 0, None) == M.MVS_ERR_ARG
    assert L.mvs_ps_run_algorithm(None) == M.MVS_ERR_ARG
    assert L.mvs_tgv2_workspace_bytes(0, 4, 1) == 0
    assert L.mvs_tgv2_sparse(8, 8, None, None, None, 5.0, 10, *([1.0] * 7), None, None, 0, None) == M.MVS_ERR_ARG
    assert L.mvs_tgv2_sparse(0, 8, *([None] * 3), 5.0, 10, *([1.0] * 7), *([None] * 2), 0, None) == M.MVS_ERR_ARG
    assert L.mvs_tgv2_sparse_workspace_bytes(0, 4) == 0
    # 8 state fields double-buffered + ref, T11, T12, T22, weights, Ds
    assert L.mvs_tgv2_sparse_workspace_bytes(640, 480) == 640 * 480 * 4 * 22
    assert L.mvs_ps_tgv_denoise_from_sparse(None, None, 1, *([1.0] * 7)) == M.MVS_ERR_ARG
    assert L.mvs_tvl1_workspace_bytes(640, 480) >= 640 * 480 * 4 * 11


def test_planesweep_handle_host_state_without_device():
    """The handle's setters and validation are host-only."""
    ps = M.PlaneSweep()
    with pytest.raises(M.MvsError):
        ps.setWindowSize(4)
    with pytest.raises(M.MvsError):
        ps.setNumberofPlanes(0)
    with pytest.raises(M.MvsError):
        ps.set_sources([np.zeros((4, 4), np.float32)], [np.eye(3)], [np.zeros(3)])   # no reference yet
    ps.set_reference(np.zeros((16, 20), np.float32), np.eye(3), np.zeros(3))
    ps.setSweepOptions(M.MOMENTS_COMPENSATED, M.SWEEP_AGGREGATED, True)
    with pytest.raises(M.MvsError):
        ps.setSweepOptions(9, 0, True)
    ps.close()
