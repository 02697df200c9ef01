"""The hybrid ph-multigrid preconditioner on the device against the
oracle's restatement of phmg_t (src/multigrid/phmg.f90) with its
Chebyshev-Jacobi smoothers and tree-AMG coarse solver.

Bars: the set-up (levels, aggregates, the 150-step power-iteration
eigenvalue estimates of every smoothed and every AMG level) to 1e-9
relative; one application to 1e-9 relative (max-norm; the device sums its
inner products and contractions in other orders, and those enter the
Chebyshev coefficients); CG, flexible CG and GMRES with phmg within +-1
iteration of the oracle and solutions to 1e-7.  Boxes with and without
deformation, periodic directions, a rotated-element mesh, and a non-default
schedule with four AMG levels."""
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


def _pair(nb, oracle, nel, lx, per=(False,) * 3, amp=0.0, hi=1.0, dirichlet=True, mesh_seed=None):
    if mesh_seed is not None:
        from neko_b200 import workloads
        ids, xyz = workloads.box_mesh(nel, rotate_seed=mesh_seed)
        P = nb.Problem.from_mesh(ids, xyz, lx, deform=amp, dirichlet=dirichlet)
        O = oracle.OracleProblem.from_elements(ids, xyz, lx)
    else:
        P = nb.Problem(nel, lx, hi=(hi,) * 3, periodic=per, deform=amp, dirichlet=dirichlet)
        O = oracle.OracleProblem.box(nel, lx, hi=(hi,) * 3, periodic=per)
    if amp:
        O.deform_sine(amp)
    O.coef()
    if dirichlet:
        O.bc_boundary()
    return P, O


CASES = [dict(nel=(4, 4, 4), lx=8),
         dict(nel=(3, 4, 3), lx=6, amp=0.05),
         dict(nel=(4, 3, 4), lx=8, per=(True, False, True), amp=0.05, hi=2 * np.pi),
         dict(nel=(3, 2, 4), lx=6, amp=0.05, mesh_seed=1)]


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("case", CASES, ids=range(len(CASES)))
def test_phmg_setup_and_apply_match_oracle(nb, oracle, case):
    P, O = _pair(nb, oracle, **case)
    H = oracle.OraclePhmg(O)
    M = nb.Phmg()
    M.init(P)
    assert int(M.describe(P, 0)) == H.levels
    for i in range(H.levels):
        assert int(M.describe(P, 1, i)) == H.level_lx(i)
    for i in range(H.levels - 1):
        lam_d, lam_o = M.describe(P, 4, i), H.cheby(i)[2]
        assert abs(lam_d - lam_o) <= 1e-9 * lam_o, (i, lam_d, lam_o)
    assert int(M.describe(P, 5)) == H.amg_levels
    for i in range(1, H.amg_levels):
        assert int(M.describe(P, 6, i)) == H.amg_nodes(i)
    for i in range(H.amg_levels):
        lam_d, lam_o = M.describe(P, 9, i), H.amg_cheby(i)[2]
        assert abs(lam_d - lam_o) <= 1e-9 * lam_o, (i, lam_d, lam_o)
    assert M.describe(P, 10) > 0
    rng = np.random.default_rng(7)
    r = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n)))
    z = P.zeros()
    M.solve(z, _cuda(r), P)
    torch.cuda.synchronize()
    assert _rel(_np(z), H.apply(r)) < 1e-9
    H.close()


@pytest.mark.parametrize("kind", ["cg", "fcg", "gmres"])
@pytest.mark.parametrize("case", [0, 2, 3])
def test_krylov_with_phmg_matches_oracle(nb, oracle, kind, case):
    P, O = _pair(nb, oracle, **CASES[case])
    H = oracle.OraclePhmg(O)
    rng = np.random.default_rng(11 + case)
    b = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n)))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    xo, it_o, _, _ = H.krylov(b, 300, 1e-9 * r0, kind=kind)
    ksp = {"cg": nb.CG, "fcg": nb.FCG, "gmres": nb.GMRES}[kind]
    x = P.zeros()
    mon = ksp(max_iter=300, abs_tol=1e-9 * r0, M=nb.Phmg()).solve(nb.AxHelm(), x, _cuda(b), P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert _rel(_np(x), xo) < 1e-7
    H.close()


def test_phmg_other_schedule_and_amg_depth(nb, oracle):
    """lx 9 -> 6 -> 3 -> 2 with two Chebyshev steps a level, four AMG levels
    (a second greedy level on aggregate adjacency), degree 3, two cycles."""
    P, O = _pair(nb, oracle, (16, 8, 4), 9, per=(True, False, False), amp=0.05, hi=2 * np.pi)
    kw = dict(smoother_iterations=2, schedule=(5, 2, 1), coarse_levels=4, coarse_iterations=2,
              cheby_degree=3)
    H = oracle.OraclePhmg(O, **kw)
    M = nb.Phmg(**kw)
    M.init(P)
    assert [int(M.describe(P, 1, i)) for i in range(4)] == [9, 6, 3, 2]
    assert int(M.describe(P, 5)) == H.amg_levels == 4
    rng = np.random.default_rng(13)
    r = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n)))
    z = P.zeros()
    M.solve(z, _cuda(r), P)
    torch.cuda.synchronize()
    assert _rel(_np(z), H.apply(r)) < 1e-9
    H.close()


def test_phmg_rejects_bad_settings(nb, oracle):
    P, _ = _pair(nb, oracle, (2, 2, 2), 5)
    for kw in (dict(schedule=(4, 1)), dict(schedule=(2, 3)), dict(schedule=(0,)),
               dict(coarse_levels=1)):
        with pytest.raises(nb.NekoB200Error) as ei:
            nb.Phmg(**kw).init(P)
        assert ei.value.status == 1
