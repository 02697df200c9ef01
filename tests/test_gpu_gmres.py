"""Device GMRES (nb_solve with NB_KSP_GMRES) against the oracle's
restatement of gmres_device_solve (src/krylov/bcknd/device/
gmres_device.F90:319-487): iteration counts within +-1, solutions within
1e-7 relative (max-norm; mean-free for the singular periodic problems).
Cases cover restarts (more iterations than m_restart), the Jacobi and hsmg
preconditioners, the h2 term and the mixed-precision hsmg."""
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


def _setup(nb, oracle, nel, lx, per, amp, hi, seed):
    from neko_b200 import workloads
    dirichlet = not all(per)
    P = nb.Problem(nel, lx, hi=(hi,) * 3, periodic=per, deform=amp, dirichlet=dirichlet)
    O = oracle.OracleProblem.box(nel, lx, hi=(hi,) * 3, periodic=per)
    if amp:
        O.deform_sine(amp)
    O.coef()
    if dirichlet:
        O.bc_boundary()
    x, y, z, B = O.f64("x"), O.f64("y"), O.f64("z"), O.f64("B")
    b = O.bc_apply(O.gs_add(workloads.periodic_box_rhs(x, y, z, B, seed)))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    return P, O, b, r0


def _cmp(xd, xo, singular):
    if singular:
        xd, xo = xd - xd.mean(), xo - xo.mean()
    return np.abs(xd - xo).max() / np.abs(xo).max()


@pytest.mark.parametrize("nel,lx,m", [((4, 4, 4), 6, 30), ((3, 4, 3), 8, 10),
                                      ((4, 3, 3), 5, 64)])
def test_gmres_jacobi_matches_oracle(nb, oracle, nel, lx, m):
    P, O, b, r0 = _setup(nb, oracle, nel, lx, (False,) * 3, 0.05, 1.0, 7)
    xo, it_o, rs_o, _ = O.gmres_jacobi(b, 1000, 1e-9 * r0, m_restart=m)
    x = P.zeros()
    mon = nb.GMRES(max_iter=1000, abs_tol=1e-9 * r0, M=nb.Jacobi(), m_restart=m).solve(
        nb.AxHelm(), x, _cuda(b), P.n, P)
    assert mon.converged
    assert abs(mon.res_start - rs_o) <= 1e-12 * rs_o
    assert abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert it_o > m  # the case crosses at least one restart
    assert _cmp(_np(x), xo, False) < 1e-7


def test_gmres_jacobi_h2(nb, oracle):
    """Helmholtz form h1 = 1.5, h2 = 20 (the implicit viscous step)."""
    P, O, b, r0 = _setup(nb, oracle, (3, 3, 4), 7, (False,) * 3, 0.03, 1.0, 9)
    P.set_coefficients(torch.full((P.n,), 1.5, dtype=torch.float64, device="cuda"),
                       torch.full((P.n,), 20.0, dtype=torch.float64, device="cuda"))
    O.set_f64("h1", np.full(P.n, 1.5))
    O.set_f64("h2", np.full(P.n, 20.0))
    O.set_ifh2(True)
    xo, it_o, _, _ = O.gmres_jacobi(b, 1000, 1e-10 * r0)
    x = P.zeros()
    mon = nb.GMRES(max_iter=1000, abs_tol=1e-10 * r0, M=nb.Jacobi()).solve(
        nb.AxHelm(), x, _cuda(b), P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert _cmp(_np(x), xo, False) < 1e-7


@pytest.mark.parametrize("nel,lx,per,amp,hi", [((4, 4, 4), 8, (True,) * 3, 0.05, 2 * np.pi),
                                               ((3, 4, 3), 6, (False,) * 3, 0.0, 1.0)])
def test_gmres_hsmg_matches_oracle(nb, oracle, nel, lx, per, amp, hi):
    P, O, b, r0 = _setup(nb, oracle, nel, lx, per, amp, hi, 3)
    H = oracle.OracleHsmg(O)
    xo, it_o, _, _ = H.gmres(b, 200, 1e-8 * r0)
    x = P.zeros()
    mon = nb.GMRES(max_iter=200, abs_tol=1e-8 * r0, M=nb.Hsmg()).solve(
        nb.AxHelm(), x, _cuda(b), P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert _cmp(_np(x), xo, all(per)) < 1e-7
    # mixed-precision hsmg inside the FP64 GMRES reaches the FP64 solution
    xm = P.zeros()
    mm = nb.GMRES(max_iter=200, abs_tol=1e-8 * r0, M=nb.Hsmg(mixed=True)).solve(
        nb.AxHelm(), xm, _cuda(b), P.n, P)
    assert mm.converged and mm.iter <= it_o + 3
    d, r = _np(xm), xo
    if all(per):
        d, r = d - d.mean(), r - r.mean()
    assert np.linalg.norm(d - r) / np.linalg.norm(r) < 1e-6


def test_gmres_max_iter_and_repeat(nb, oracle):
    """A budget smaller than needed stops at max_iter unconverged; a second
    solve on the same workspace (graph replayed) gives the same result."""
    P, O, b, r0 = _setup(nb, oracle, (3, 3, 3), 6, (False,) * 3, 0.0, 1.0, 2)
    S = nb.GMRES(max_iter=12, abs_tol=1e-12 * r0, M=nb.Jacobi(), m_restart=5)
    x, fb = P.zeros(), _cuda(b)
    m1 = S.solve(nb.AxHelm(), x, fb, P.n, P)
    x1 = x.clone()
    m2 = S.solve(nb.AxHelm(), x, fb, P.n, P)
    assert m1.iter == 12 and not m1.converged
    xo, it_o, _, rf = O.gmres_jacobi(b, 12, 1e-12 * r0, m_restart=5)
    assert it_o == 12
    assert torch.equal(x1, x) and m1.res_final == m2.res_final
    assert _cmp(_np(x1), xo, False) < 1e-9


@pytest.mark.parametrize("nel,lx,h2", [((4, 4, 4), 6, 0.0), ((3, 4, 3), 8, 25.0)])
def test_pipecg_jacobi_matches_oracle(nb, oracle, nel, lx, h2):
    """Pipelined CG (NB_KSP_PIPECG) against the oracle's restatement of
    pipecg_device_solve: iterations within +-1, solution 1e-7."""
    P, O, b, r0 = _setup(nb, oracle, nel, lx, (False,) * 3, 0.05, 1.0, 11)
    if h2:
        P.set_coefficients_const(1.0, h2)
        O.set_f64("h2", np.full(P.n, h2))
        O.set_ifh2(True)
    xo, it_o, rs_o, _ = O.pipecg_jacobi(b, 2000, 1e-10 * r0)
    x = P.zeros()
    mon = nb.PipeCG(max_iter=2000, abs_tol=1e-10 * r0, M=nb.Jacobi()).solve(
        nb.AxHelm(), x, _cuda(b), P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert abs(mon.res_start - rs_o) <= 1e-12 * rs_o
    assert _cmp(_np(x), xo, False) < 1e-7
