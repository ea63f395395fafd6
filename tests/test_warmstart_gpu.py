"""What the trained warm-start network gains over TGV2 without it.

On held-out seeded scenes of the full-size configuration (640x480, 8 views,
256 inverse-depth planes, 9x9 window; the network was trained on other
seeds), TGV2 runs to relative energy change 1e-4 (cap 500) once from the
winner-take-all depth (plain) and once from the network's prediction (warm),
both linearised at the winner-take-all depth so they minimise the same
energy.  The warm run must end at an energy no higher than the plain run's
(0.5% slack per frame), get below the plain run's final energy in a fraction
of its iterations, and take less device time including the network.

The speed claim is made at equal energy: the warm run reaches the plain run's
final energy at least 3x sooner (network included).  To the tolerance (the
mean relative energy change per 10 iterations over the last 50 at most 1e-4)
both runs stop where their energy flattens, the warm one lower: there the warm
runs need only take less time in total."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_warm_start_beats_plain_tgv2(cuda):
    from mvs_b200 import warmstart as WS
    params, norm, meta = WS.load_weights()
    rows = WS.evaluate([910001, 910002, 910003], WS.FrameConfig(), params, norm, device=cuda)
    for r in rows:
        assert r["warm_energy"] <= r["plain_energy"] * 1.005, r
        assert r["warm_iters_to_plain_energy"] is not None, r
        assert r["warm_err"] <= r["plain_err"] * 1.2, r
    # the network's prediction alone is already within a few percent of (often
    # below) the plain run's final energy; the winner-take-all start of the
    # plain run sits tens of percent above it
    assert np.median([r["start_energy"] / r["plain_energy"] for r in rows]) < 1.10
    reach = np.median([r["warm_iters_to_plain_energy"] for r in rows])
    plain_it = np.median([r["plain_iters"] for r in rows])
    assert reach * 3 <= plain_it, (reach, plain_it)
    plain_ms = np.mean([r["plain_ms"] for r in rows])
    to_plain_energy = plain_ms / np.mean([r["warm_ms_to_plain_energy"] for r in rows])
    assert to_plain_energy >= 3.0, to_plain_energy
    to_tolerance = plain_ms / np.mean([r["warm_ms"] for r in rows])
    assert to_tolerance > 1.0, to_tolerance
