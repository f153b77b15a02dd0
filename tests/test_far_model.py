"""The fast walk's far-cell expansion, restated in far_model.py in the
kernel's expressions: it is the monopole field's Taylor expansion to second
order about the group centre, and its error at an offset delta is bounded by
the on-axis remainder 1/(1-e)^2 - (1 + 2e + 3e^2), e = |delta| / d, of the
field at the centre (leading term 4 e^3; 9.0 % at the walk's FAR_RATIO of 4,
where a target lies at most h from the centre and the cell at least 4 h).
This test found the first build's second-derivative coefficients off by a
factor 1 / r^2."""
import numpy as np
import pytest

import far_model as fm


def _unit(rng):
    v = rng.normal(size=3)
    return v / np.linalg.norm(v)


def _remainder(e):
    return 1.0 / (1.0 - e) ** 2 - (1.0 + 2.0 * e + 3.0 * e * e)


def test_expansion_at_the_centre_is_the_field():
    rng = np.random.default_rng(5)
    src = [tuple(rng.normal(size=3) * 10.0) + (float(q),) for q in rng.choice([-3.0, -1.0, 1.0, 2.0], 20)]
    acc = fm.expansion((0.0, 0.0, 0.0), src)
    assert np.allclose(fm.evaluate(acc, (0.0, 0.0, 0.0)), fm.direct((0.0, 0.0, 0.0), src), rtol=1e-13, atol=0)


def test_gradient_and_curvature_terms_match_finite_differences():
    """J is the field's gradient and H its second derivatives at the centre:
    central differences of the exact field agree, and the trace-free
    components the kernel drops are what Laplace's equation gives."""
    s = [(3.0, -2.0, 4.5, 1.7)]
    acc = fm.expansion((0.0, 0.0, 0.0), s)
    h = 1e-4
    J = np.zeros((3, 3))
    for b in range(3):
        e = np.zeros(3)
        e[b] = h
        J[:, b] = (fm.direct(e, s) - fm.direct(-e, s)) / (2 * h)
    assert np.allclose([J[0, 0], J[1, 1], J[0, 1], J[0, 2], J[1, 2]],
                       [acc["jxx"], acc["jyy"], acc["jxy"], acc["jxz"], acc["jyz"]], rtol=1e-6)
    assert abs(np.trace(J)) < 1e-8 * np.abs(J).max()
    # second derivative of E_x along x and of E_z along x, y
    d2 = lambda a, u, v: (fm.direct(u + v, s)[a] - fm.direct(u - v, s)[a] - fm.direct(v - u, s)[a]
                          + fm.direct(-u - v, s)[a]) / (4 * h * h)
    ex_, ey_, ez_ = np.eye(3) * h
    assert np.isclose(d2(0, ex_, ex_), acc["hxxx"], rtol=1e-4)
    assert np.isclose(d2(2, ex_, ey_), acc["hxyz"], rtol=1e-4)
    assert np.isclose(d2(1, ex_, ex_), acc["hxxy"], rtol=1e-4)


@pytest.mark.parametrize("e", [1 / 8, 1 / 6, 1 / 4])
def test_error_within_the_on_axis_remainder(e):
    rng = np.random.default_rng(int(1 / e))
    worst = 0.0
    for _ in range(3000):
        d = rng.uniform(0.5, 5.0)
        u = _unit(rng)
        s = [(-d * u[0], -d * u[1], -d * u[2], 1.0)]
        delta = e * d * _unit(rng)
        acc = fm.expansion((0.0, 0.0, 0.0), s)
        err = np.linalg.norm(fm.evaluate(acc, delta) - fm.direct(delta, s)) * d * d
        worst = max(worst, err)
        assert err <= _remainder(e) * (1 + 1e-9) + 1e-12
    # the bound is reached towards the source
    assert worst > 0.95 * _remainder(e)


def test_error_is_third_order():
    s = [(2.0, 1.0, -3.0, 1.0)]
    acc = fm.expansion((0.0, 0.0, 0.0), s)
    v = np.array([0.3, -0.5, 0.8])
    v /= np.linalg.norm(v)
    errs = [np.linalg.norm(fm.evaluate(acc, t * v) - fm.direct(t * v, s)) for t in (0.04, 0.02, 0.01)]
    for a, b in zip(errs, errs[1:]):
        assert 7.0 < a / b < 9.0


def test_far_cells_of_a_group_add():
    """Many far cells folded into one expansion: the group's error is at most
    the sum of each cell's bound, with every cell at least 4 h from the
    centre and every target within h of it."""
    rng = np.random.default_rng(11)
    h = 0.05
    src, bound = [], 0.0
    for _ in range(200):
        d = rng.uniform(4 * h, 40 * h)
        u = _unit(rng)
        q = float(rng.choice([-2.0, -1.0, 1.0, 3.0]))
        src.append((d * u[0], d * u[1], d * u[2], q))
        bound += abs(q) / d ** 2 * _remainder(h / d)
    acc = fm.expansion((0.0, 0.0, 0.0), src)
    for _ in range(50):
        delta = h * rng.uniform(0, 1) * _unit(rng)
        assert np.linalg.norm(fm.evaluate(acc, delta) - fm.direct(delta, src)) <= bound * (1 + 1e-9)
