"""CPU checks of the oracle's full-stress operator and coupled CG (no GPU):
the operator is symmetric and positive semi-definite, the rigid motions are
in its kernel, and the coupled CG drives the assembled residual down."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def O(oracle):
    P = oracle.OracleProblem.box((3, 2, 2), 6)
    P.deform_sine(0.05)
    P.coef()
    P.bc_boundary()
    return P


def test_stress_operator_symmetric_psd(O):
    rng = np.random.default_rng(0)
    a = [rng.standard_normal(O.n) for _ in range(3)]
    b = [rng.standard_normal(O.n) for _ in range(3)]
    Aa, Ab = O.ax_helm_stress(*a), O.ax_helm_stress(*b)
    ab = sum(np.dot(x, y) for x, y in zip(Aa, b))
    ba = sum(np.dot(x, y) for x, y in zip(Ab, a))
    assert abs(ab - ba) <= 1e-12 * max(abs(ab), 1.0)
    assert sum(np.dot(x, y) for x, y in zip(Aa, a)) > 0


def test_stress_operator_rigid_motions(O):
    x, y, z = O.f64("x"), O.f64("y"), O.f64("z")
    one, zero = np.ones(O.n), np.zeros(O.n)
    scale = max(np.abs(c).max() for c in O.ax_helm_stress(x, y, z))
    for f in ((one, zero, zero), (zero, zero, one), (-y, x, zero), (z, zero, -x)):
        assert max(np.abs(c).max() for c in O.ax_helm_stress(*f)) < 1e-12 * scale


def test_coupled_cg_converges(O):
    rng = np.random.default_rng(1)
    f = [O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n))) for _ in range(3)]
    (x, y, z), it, r0, r1 = O.cg_coupled(f, 2000, 1e-9, stress=True, jacobi=True)
    assert 0 < it < 2000 and r1 < 1e-9
    # the residual of the assembled, masked system is small
    res = [O.bc_apply(O.gs_add(a)) for a in O.ax_helm_stress(x, y, z)]
    err = max(np.abs(res[c] - f[c]).max() for c in range(3))
    assert err < 1e-6 * max(np.abs(c).max() for c in f)
