"""mvs_tgv2_run_warm: the warm-start entry point against the plain run.

* started where the plain run starts (u = u_lin, v = 0, duals at zero) it is
  the plain run, bit for bit;
* restarted from the plain run's own state after k iterations, its starting
  energy is the plain run's energy at k (same linearisation point), and its
  returned v is the state it was given when it runs no iteration."""
import numpy as np
import pytest

import mvs_b200 as M
from mvs_b200 import hostmath as hm, scenes

pytestmark = pytest.mark.gpu


def _setup(cuda):
    import torch
    fr, planes, win = scenes.config_tiny(seed=6, width=96, height=64, n_src=3, n_planes=16, win=5)
    K = np.float32(fr.ref_cam.K_1based)
    rel = [hm.relative_f32(fr.ref_cam.R, fr.ref_cam.t, c.R, c.t) for c in fr.src_cams]
    Rs = np.stack([r[0].reshape(9) for r in rel])
    ts = np.stack([r[1] for r in rel])
    iK = hm.inv3_f32(K)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(cuda)
    rng = np.random.default_rng(6)
    start = fr.depth_gt * (1 + 0.05 * rng.standard_normal(fr.depth_gt.shape))
    h, w = fr.ref.shape
    ws = torch.empty(M.tgv2_workspace_bytes(w, h, 3) // 8 + 1, dtype=torch.int64, device=cuda)
    return dict(ref=T(fr.ref), srcs=T(np.stack(fr.srcs)), K=K.reshape(9), iK=iK.reshape(9), Rs=Rs, ts=ts,
                start=T(start), ws=ws, h=h, w=w)


def test_warm_from_plain_start_is_plain(cuda):
    import torch
    s = _setup(cuda)
    prm = M.tgv2_params(niters=200, warps=1, tol=1e-3, check_every=10)
    u1 = s["start"].clone()
    it1, e1 = M.tgv2_run(s["ref"], s["srcs"], s["K"], s["iK"], s["Rs"], s["ts"], prm, u1, u_from_input=True,
                         workspace=s["ws"])
    u2 = s["start"].clone()
    v2 = torch.zeros((2, s["h"], s["w"]), device=cuda)
    it2, e2 = M.tgv2_run_warm(s["ref"], s["srcs"], s["K"], s["iK"], s["Rs"], s["ts"], prm, s["start"], u2, v2,
                              dual_sigma=0.0, workspace=s["ws"])
    torch.cuda.synchronize()
    assert it1 == it2 and e1 == e2
    assert torch.equal(u1, u2)


def test_warm_restart_energy_and_v(cuda):
    import torch
    s = _setup(cuda)
    prm = M.tgv2_params(niters=60, warps=1, tol=0.0)
    u = s["start"].clone()
    v = torch.zeros((2, s["h"], s["w"]), device=cuda)
    it, e60 = M.tgv2_run_warm(s["ref"], s["srcs"], s["K"], s["iK"], s["Rs"], s["ts"], prm, s["start"], u, v,
                              workspace=s["ws"])
    assert it == 60 and float(v.abs().max()) > 0
    # zero iterations from that state: same energy, v handed back unchanged
    u2, v2 = u.clone(), v.clone()
    p0 = M.tgv2_params(niters=0, warps=1, tol=0.0)
    it0, e0 = M.tgv2_run_warm(s["ref"], s["srcs"], s["K"], s["iK"], s["Rs"], s["ts"], p0, s["start"], u2, v2,
                              dual_sigma=10.0, workspace=s["ws"])
    torch.cuda.synchronize()
    assert it0 == 0
    assert e0 == e60
    assert torch.equal(u2, u) and torch.equal(v2, v)
    # continuing from the state with dual start: the energy keeps going down
    u3, v3 = u.clone(), v.clone()
    p40 = M.tgv2_params(niters=40, warps=1, tol=0.0)
    _, e3 = M.tgv2_run_warm(s["ref"], s["srcs"], s["K"], s["iK"], s["Rs"], s["ts"], p40, s["start"], u3, v3,
                            dual_sigma=10.0, workspace=s["ws"])
    assert np.isfinite(e3) and e3 < e60 * 1.001
