"""GPU parity of the hsmg preconditioner and the flexible CG that drives it,
against the CPU oracle (hsmg_solve, CPU branch, src/krylov/pc_hsmg.f90).

Tolerances: one preconditioner application agrees to 1e-10 relative
(max-norm): the FDM factors come from different eigensolvers (signs of the
eigenvectors may differ; S D^-1 S' does not) and the coarse level runs ten
CG iterations that amplify rounding.  Solves: iteration counts within +-1,
solutions to 1e-7 relative.
"""
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


CASES = [((4, 4, 4), 8, (False,) * 3, 0.0, 1.0),
         ((3, 4, 3), 6, (False,) * 3, 0.0, 1.0),
         ((4, 4, 4), 8, (True,) * 3, 0.05, 2 * np.pi),
         ((3, 3, 4), 10, (True, False, True), 0.05, 2 * np.pi),
         ((3, 3, 3), 5, (True,) * 3, 0.05, 2 * np.pi),
         ((3, 3, 3), 4, (False,) * 3, 0.0, 1.0)]


def _pair(nb, oracle, nel, lx, per, amp, hi):
    dirichlet = not all(per)
    P = nb.Problem(nel, lx, hi=(hi,) * 3, periodic=per, deform=amp, dirichlet=dirichlet)
    O = oracle.OracleProblem.box(nel, lx, hi=(hi,) * 3, periodic=per)
    if amp:
        O.deform_sine(amp)
    O.coef()
    if dirichlet:
        O.bc_boundary()
    return P, O


@pytest.mark.parametrize("nel,lx,per,amp,hi", CASES)
def test_hsmg_apply_matches_oracle(nb, oracle, nel, lx, per, amp, hi):
    P, O = _pair(nb, oracle, nel, lx, per, amp, hi)
    H = oracle.OracleHsmg(O)
    rng = np.random.default_rng(lx)
    r = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(P.n)))
    if all(per):
        r -= r.sum() / r.size  # consistent right-hand side of a singular problem
        r = O.gs_add(r * O.f64("mult"))
    ref = H.apply(r)
    # Fully periodic problems have a singular coarse level; on very small
    # meshes its ten CG iterations amplify rounding by orders of magnitude.
    # The bound is then ten times the oracle's own change under a 1e-15
    # relative perturbation of r.
    tol = 1e-10
    if all(per):
        rp = r * (1 + 1e-15 * rng.standard_normal(r.size))
        sens = np.abs(H.apply(rp) - ref).max() / np.abs(ref).max()
        tol = max(tol, 10 * sens)
    z = P.zeros()
    nb.Hsmg().solve(z, _cuda(r), P)
    torch.cuda.synchronize()
    err = np.abs(_np(z) - ref).max() / np.abs(ref).max()
    assert err < tol, (err, tol)


@pytest.mark.parametrize("nel,lx,per,amp,hi", CASES[:4])
def test_fcg_hsmg_matches_oracle(nb, oracle, nel, lx, per, amp, hi):
    from neko_b200 import workloads
    P, O = _pair(nb, oracle, nel, lx, per, amp, hi)
    H = oracle.OracleHsmg(O)
    x, y, z, B = O.f64("x"), O.f64("y"), O.f64("z"), O.f64("B")
    b = O.gs_add(workloads.config2_rhs_local(x, y, z, B, 3))
    b = O.bc_apply(b)
    mult = O.f64("mult")
    r0 = np.sqrt(np.sum(b * mult * b) / O.volume)
    xo, it_o, rs_o, rf_o = H.cg(b, 200, 1e-8 * r0, flexible=True)
    xd = P.zeros()
    mon = nb.FCG(max_iter=200, abs_tol=1e-8 * r0, M=nb.Hsmg()).solve(nb.AxHelm(), xd, _cuda(b),
                                                                     P.n, P)
    assert mon.converged
    assert abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    xdn = _np(xd)
    if all(per):  # solutions of the singular problem agree up to a constant
        xdn, xo = xdn - xdn.mean(), xo - xo.mean()
    assert np.abs(xdn - xo).max() / np.abs(xo).max() < 1e-7


def test_hsmg_rejects_bad_lx(nb):
    P = nb.Problem((3, 3, 3), 16)
    z = P.zeros()
    with pytest.raises(nb.NekoB200Error):
        nb.Hsmg().solve(z, P.zeros(), P)
