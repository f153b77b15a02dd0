"""The non-allocating field query (pot_gpu_field_at_noalloc) against the
allocating one (pot_gpu_field_at), through the C ABI.

The variant exists for callers that must not allocate device memory while
they run; it stages its work in one fixed device array instead.  Its results
must match pot_gpu_field_at's for the same tree and points, call after call
(the array keeps the previous call's contents), in the plain FP64 form and
in the FP32 fast form.  This file sorts last so that a run stopping at the
first failure has already run every other test.
"""
import numpy as np
import pytest

from common import SMALL, oracle_snapshot, run_config
from pot_b200.gpu import NOALLOC_MAX_POINTS, PotError, Run

pytestmark = pytest.mark.gpu


def _points(o, rng, k):
    P = o.particles()
    idx = np.sort(rng.choice(np.arange(1, len(P)), size=k, replace=False)).astype(np.uint32)
    xyz = np.stack([P["x"][idx], P["y"][idx], P["z"][idx]], 1) + rng.normal(0, 1e-10, (k, 3))
    return idx, xyz


@pytest.mark.parametrize("form,leaf", [("plain", 0), ("fast", 16)])
def test_noalloc_matches_allocating_query_twice(form, leaf):
    d = dict(SMALL, N=30001)
    o = oracle_snapshot(d, seed=6, mode="gpu")
    o.set_grain(q=-300)
    P = o.particles()
    g = dict(q=-300, pos=(P[0]["x"], P[0]["y"], P[0]["z"]))
    rng = np.random.default_rng(17)
    with Run(run_config(d), form=form, leaf_size=leaf, seed=6) as r:
        r.upload(P, g)
        r.build_tree()
        for k in (4000, 1500):  # two calls in a row, the second smaller
            idx, xyz = _points(o, rng, k)
            want = r.field_at(idx, xyz)
            got = r.field_at_noalloc(idx, xyz)
            mag = np.sqrt((want ** 2).sum(1))
            assert np.all(np.isfinite(got))
            assert np.max(np.abs(got - want).max(1) / mag) < 1e-12


@pytest.mark.parametrize("form,leaf", [("plain", 0), ("fast", 16)])
def test_noalloc_first_on_a_fresh_run_allocates_nothing(form, leaf):
    """On a run that has never answered a field query (no query buffers
    exist yet), two no-alloc calls leave the device's free memory as it was;
    the allocating query afterwards gives the same fields."""
    import torch
    d = dict(SMALL, N=30001)
    o = oracle_snapshot(d, seed=8, mode="gpu")
    o.set_grain(q=-250)
    P = o.particles()
    g = dict(q=-250, pos=(P[0]["x"], P[0]["y"], P[0]["z"]))
    rng = np.random.default_rng(23)
    pts = [_points(o, rng, k) for k in (3000, 2000)]
    # another run answers one query first, so that every kernel the query
    # uses is already loaded on the device (module loading is not the call's)
    with Run(run_config(d), form=form, leaf_size=leaf, seed=8) as w:
        w.upload(P, g)
        w.build_tree()
        w.field_at(*pts[1])
        w.field_at_noalloc(*pts[1])
    torch.cuda.synchronize()
    with Run(run_config(d), form=form, leaf_size=leaf, seed=8) as r:
        r.upload(P, g)
        r.build_tree()
        r.sync()
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        got = [r.field_at_noalloc(idx, xyz) for idx, xyz in pts]
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        assert free1 >= free0, "the no-alloc query took %d bytes of device memory" % (free0 - free1)
        for (idx, xyz), e in zip(pts, got):
            want = r.field_at(idx, xyz)
            mag = np.sqrt((want ** 2).sum(1))
            assert np.all(np.isfinite(e))
            assert np.max(np.abs(e - want).max(1) / mag) < 1e-12


def test_noalloc_rejects_oversized_requests():
    d = dict(SMALL, N=2049)
    o = oracle_snapshot(d, seed=6, mode="gpu")
    with Run(run_config(d), seed=6) as r:
        r.upload(o.particles())
        r.build_tree()
        n = NOALLOC_MAX_POINTS + 1
        with pytest.raises(PotError) as e:
            r.field_at_noalloc(np.ones(n, np.uint32), np.full((n, 3), 7.0e-7))
        assert e.value.status == -11
