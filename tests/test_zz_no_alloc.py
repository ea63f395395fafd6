"""The allocation-free sweep entry point (mvs_sweep_noalloc) through the C ABI.

It serves callers that cannot allocate device memory while they run (plugin
hosts that fix a library's memory at start-up, real-time loops): its scratch
is a fixed array inside the library.  Checked against mvs_sweep with a caller
workspace, on calls in a row (the shared array keeps the previous call's
contents, which must not leak into the next result).  This file is collected
last, so a stop-at-first-failure run has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import mvs_b200 as M
from mvs_b200 import scenes

pytestmark = pytest.mark.gpu


def _inputs(cuda, seed, w, h, n_src, n_planes, win):
    import torch
    fr, planes, _ = scenes.config_tiny(seed=seed, width=w, height=h, n_src=n_src, n_planes=n_planes, win=win)
    d = dict(ref=torch.from_numpy(fr.ref).to(cuda), srcs=torch.from_numpy(np.stack(fr.srcs)).to(cuda),
             depths=torch.from_numpy(planes).to(cuda))
    rel = [M.relative_pose(fr.ref_cam.R, fr.ref_cam.t, c.R, c.t) for c in fr.src_cams]
    return fr, planes, d, rel


def _outputs(cuda, desc, n_lab):
    import torch
    h, w = desc.height, desc.width
    return dict(depth=torch.full((h, w), -7.0, device=cuda),
                labels=torch.full((n_lab, h, w), -7, dtype=torch.int32, device=cuda),
                best=torch.full((n_lab, h, w), -7.0, device=cuda),
                cost=(torch.zeros((desc.n_planes, h, w), dtype=torch.int16, device=cuda)
                      if desc.mode == M.SWEEP_AGGREGATED else None))


def _call(L, fn, desc, d, H, o, extra):
    p = M._ptr
    args = [C.byref(desc), p(d["ref"]), p(d["srcs"]), p(H), p(d["depths"]), p(o["depth"]), p(o["labels"]),
            p(o["best"]), p(o["cost"])]
    return getattr(L, fn)(*args, *extra)


@pytest.mark.parametrize("mode,moments", [(M.SWEEP_PER_VIEW, M.MOMENTS_REFERENCE),
                                          (M.SWEEP_AGGREGATED, M.MOMENTS_COMPENSATED)])
def test_noalloc_matches_workspace_entry_point_twice(cuda, mode, moments):
    """Three calls in a row on frames of one size with different content: 24
    planes (one plane chunk: every scratch word written directly), 300 planes
    (many chunks merged in the scratch, which the call clears first), then 24
    planes again.  Each must equal mvs_sweep with a fresh caller workspace bit
    for bit, so nothing of the previous call's scratch reaches a result."""
    import torch
    L = M.lib()
    w, h, v = 96, 72, 3
    for seed, p in [(31, 24), (32, 300), (33, 24)]:
        fr, planes, d, rel = _inputs(cuda, seed, w, h, v, p, 7)
        desc = M.sweep_desc(w, h, v, len(planes), 7, moments, mode, 1e-4, 0.5, 5.0)
        H = torch.empty(v * len(planes) * 9, device=cuda)
        M.sweep_homographies(desc, fr.ref_cam.K_1based, rel, d["depths"], H)
        n_lab = v if mode == M.SWEEP_PER_VIEW else 1
        want = _outputs(cuda, desc, n_lab)
        ws = torch.empty(M.sweep_workspace_bytes(desc) // 8 + 1, dtype=torch.int64, device=cuda)
        rc = _call(L, "mvs_sweep", desc, d, H, want, [M._ptr(ws), ws.numel() * 8, None])
        assert rc == 0, L.mvs_last_error()
        got = _outputs(cuda, desc, n_lab)
        rc = _call(L, "mvs_sweep_noalloc", desc, d, H, got, [None])
        assert rc == 0, L.mvs_last_error()
        assert L.mvs_last_error() == b""
        torch.cuda.synchronize()
        for k in ("depth", "labels", "best", "cost"):
            if want[k] is not None:
                np.testing.assert_array_equal(got[k].cpu().numpy(), want[k].cpu().numpy())
        assert (got["labels"].cpu().numpy() >= 0).mean() > 0.5


def test_noalloc_rejects_sweeps_beyond_the_fixed_scratch(cuda):
    L = M.lib()
    cap = L.mvs_sweep_noalloc_scratch_bytes()
    assert cap == 32 << 20
    # 640x480 with 16 views needs 640*480*16*8 bytes > 32 MiB
    desc = M.sweep_desc(640, 480, 16, 8, 9)
    dummy = C.c_void_p(1)
    rc = L.mvs_sweep_noalloc(C.byref(desc), dummy, dummy, dummy, dummy, dummy, None, None, None, None)
    assert rc == M.MVS_ERR_ARG
    assert b"scratch" in L.mvs_last_error()
