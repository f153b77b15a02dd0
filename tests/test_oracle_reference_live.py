"""The oracle against the reference program compiled here (skipped where
the reference tree is absent, e.g. on a GPU box without oracle/_ref)."""
import numpy as np
import pytest

from common import SMALL, STRESS, params
from oracle.oracle import Oracle, RefLib


def _ref(variant):
    try:
        return RefLib(variant, build=True)
    except Exception as e:  # reference sources not present
        pytest.skip("reference not available: %s" % e)


@pytest.mark.parametrize("variant,d,seed,steps", [("sceptic", STRESS, 3, 40), ("sphere", STRESS, 4, 40),
                                                  ("sceptic", dict(SMALL, N=2049, theta=0.8), 5, 30)])
def test_reference_mode_bit_identical(variant, d, seed, steps):
    ref = _ref(variant).setup(params(d), seed=seed)
    o = Oracle(params(d), mode="reference", sceptic=variant == "sceptic", seed=seed)
    for _ in range(steps):
        ref.step()
        o.step()
    a, b = ref.particles(), o.particles()
    a["_pad"] = 0
    b["_pad"] = 0
    assert a.tobytes() == b.tobytes()
    ga, gb = ref.grain(), o.grain()
    for k in ("q", "m", "tot_absor_e", "t_steps", "chi_b"):
        assert ga[k] == gb[k], k


def test_gpu_semantics_close_to_reference():
    """The GPU-semantics step (every target sees pre-step sources) differs
    from the reference's in-place half-drift only at O(v dt) in the sources:
    one step from the same state agrees to a small fraction of the spacing."""
    d = dict(SMALL, N=4097)
    ref = _ref("sceptic").setup(params(d), seed=2)
    o = Oracle(params(d), mode="gpu", seed=2, init=False)
    o.set_particles(ref.particles())
    ref.step()
    o.step()
    a, b = ref.particles(), o.particles()
    moved = (a["species"] == 2)
    R = d["r"] * d["mpp"]
    # electrons: same push except the sources' half-drift; reinjected ones differ (RNG)
    dx = np.sqrt((a["x"] - b["x"]) ** 2 + (a["y"] - b["y"]) ** 2 + (a["z"] - b["z"]) ** 2)[moved]
    assert np.median(dx) < 1e-7 * R
