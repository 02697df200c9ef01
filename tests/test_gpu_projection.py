"""The pressure-solve caller's steps around nb_solve: solution-space
projection (projection_t, src/common/projection.f90) and the mean removal of
a singular problem (device_ortho, src/math/operators.f90:349-368), against
the oracle's restatement of the device forms.

A sequence of time steps with slowly changing right-hand sides: project_on,
solve, project_back, as fluid_pnpn.f90:812-866 does (activation from the
first step here).  Bars: the basis size equal to the oracle's at every step,
iteration counts within +-1, solutions within 1e-7 relative (max-norm), the
projected right-hand side's norm within 1e-6 of the oracle's."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import neko_b200
    neko_b200.load()
    return neko_b200


def _np(t):
    return t.detach().cpu().numpy()


def _cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


@pytest.mark.parametrize("pc,L", [("jacobi", 4), ("hsmg", 3)])
def test_projection_sequence_matches_oracle(nb, oracle, pc, L):
    nel, lx = (4, 3, 4), 6
    P = nb.Problem(nel, lx, deform=0.05)
    O = oracle.OracleProblem.box(nel, lx)
    O.deform_sine(0.05)
    O.coef()
    O.bc_boundary()
    H = oracle.OracleHsmg(O) if pc == "hsmg" else None
    J = nb.Projection(P, L=L, activ_step=0)
    Jo = oracle.OracleProjection(O, L)
    rng = np.random.default_rng(12)
    mult = O.f64("mult")
    base = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n)))
    for t in range(1, 9):
        noise = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n)))
        b = base * (1 + 0.1 * t) + 0.01 * noise
        r0 = np.sqrt(np.sum(b * mult * b) / O.volume)
        tol = 1e-10 * r0
        # oracle step
        bpo = Jo.project_on(b)
        if H is None:
            xo, it_o, _, _ = O.cg_jacobi(bpo, 2000, tol)
        else:
            xo, it_o, _, _ = H.cg(bpo, 200, tol, flexible=True)
        xo = Jo.project_back(xo)
        # device step
        bd = _cuda(b)
        J.pre_solving(bd, t)
        x = P.zeros()
        solver = (nb.CG(max_iter=2000, abs_tol=tol, M=nb.Jacobi()) if H is None else
                  nb.FCG(max_iter=200, abs_tol=tol, M=nb.Hsmg()))
        mon = solver.solve(nb.AxHelm(), x, bd, P.n, P)
        J.post_solving(x, t)
        m, pm, pres = J.info()
        assert m == Jo.m, (t, m, Jo.m)
        assert abs(mon.iter - it_o) <= 1, (t, mon.iter, it_o)
        rpo = np.sqrt(np.sum(bpo * mult * bpo) / O.volume)
        rpd = np.sqrt(float((bd * P.field("mult") * bd).sum()) / P.volume)
        assert abs(rpd - rpo) <= 1e-6 * rpo + 1e-12 * r0, (t, rpd, rpo)
        xd = _np(x)
        assert np.abs(xd - xo).max() / np.abs(xo).max() < 1e-7, t
        if t > 1:
            assert rpo < 0.1 * r0  # the projection removed most of the right-hand side
    J.close()


def test_projection_reorthogonalize_and_clear(nb):
    """After new coefficients, reorthogonalize rebuilds B = A X so the
    projection of A x_k recovers x_k; clear empties the basis."""
    P = nb.Problem((3, 3, 3), 6, deform=0.02)
    J = nb.Projection(P, L=3, activ_step=0)
    rng = np.random.default_rng(4)
    xs = []
    for _ in range(2):
        f = P.zeros()
        f.copy_(_cuda(rng.standard_normal(P.n)))
        P.gs.op(f)
        P.bclst.apply(f)
        J.project_on(f)
        x = P.zeros()
        nb.CG(max_iter=2000, abs_tol=1e-12, M=nb.Jacobi()).solve(nb.AxHelm(), x, f, P.n, P)
        J.project_back(x)
        xs.append(x.clone())
    P.set_coefficients(torch.full((P.n,), 2.0, dtype=torch.float64, device="cuda"))
    J.reortho_basis()
    # b = A x_0 with the new operator: the projection recovers x_0
    b = P.zeros()
    nb.AxHelm().compute(b, xs[0], P)
    P.gs.op(b)
    P.bclst.apply(b)
    b0 = b.clone()
    J.project_on(b)
    x = P.zeros()
    J.project_back(x)  # x = xbar, which then enters the basis (dependent: dropped)
    torch.cuda.synchronize()
    assert float((x - xs[0]).abs().max() / xs[0].abs().max()) < 1e-9
    assert float(b.abs().max()) < 1e-9 * float(b0.abs().max())
    J.clear()
    assert J.info()[0] == 0


def test_ortho_removes_mean(nb):
    P = nb.Problem((3, 3, 3), 5, periodic=(True,) * 3, hi=(6.0,) * 3, dirichlet=False)
    rng = np.random.default_rng(6)
    v = rng.standard_normal(P.n) + 3.0
    x = _cuda(v)
    nb.ortho(x, P)
    torch.cuda.synchronize()
    ref = v - v.sum() / v.size
    assert np.abs(_np(x) - ref).max() < 1e-13
