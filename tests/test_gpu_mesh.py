"""Problems built from a caller's unstructured hexahedral mesh
(nb_problem_create_mesh) against the oracle's mesh path (mesh_t, dofmap_t,
gs_init_mapping, coef_t on the same vertex ids and coordinates).

Meshes: a box whose elements' local frames are turned by random cube
rotations, so neighbours meet with arbitrary relative orientation.  Bars as
for the box: geometric factors 1e-12 of their scale, ax_helm 1e-12, gather-
scatter bit-exact, Jacobi-PCG / GMRES / hsmg-FCG iterations within +-1 and
solutions 1e-7, one hsmg apply 1e-10."""
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


def _pair(nb, oracle, nel, lx, seed, deform):
    from neko_b200 import workloads
    ids, xyz = workloads.box_mesh(nel, rotate_seed=seed)
    P = nb.Problem.from_mesh(ids, xyz, lx, deform=deform, dirichlet=True)
    O = oracle.OracleProblem.from_elements(ids, xyz, lx)
    if deform:
        O.deform_sine(deform)
    O.coef()
    O.bc_boundary()
    return P, O


@pytest.mark.parametrize("nel,lx,seed,deform", [((3, 2, 4), 6, 1, 0.05), ((4, 3, 3), 8, 2, 0.0),
                                                ((2, 3, 2), 5, 3, 0.05), ((3, 3, 3), 10, 4, 0.05)])
def test_rotated_mesh_matches_oracle(nb, oracle, nel, lx, seed, deform):
    P, O = _pair(nb, oracle, nel, lx, seed, deform)
    for name in ("x", "y", "z", "g11", "g22", "g33", "g12", "g13", "g23", "B", "mult"):
        a, b = _np(P.field(name)), O.f64(name)
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1.0), name
    rng = np.random.default_rng(lx)
    u = rng.uniform(-1, 1, P.n)
    w = P.zeros()
    nb.AxHelm().compute(w, _cuda(u), P)
    torch.cuda.synchronize()
    ref = O.ax_helm(u)
    assert np.abs(_np(w) - ref).max() / np.abs(ref).max() < 1e-12
    g = _cuda(u)
    P.gs.op(g)
    torch.cuda.synchronize()
    assert np.array_equal(_np(g), O.gs_add(u))
    # Jacobi-PCG
    b = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(P.n)))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    xo, it_o, _, _ = O.cg_jacobi(b, 2000, 1e-10 * r0)
    x = P.zeros()
    mon = nb.CG(max_iter=2000, abs_tol=1e-10 * r0, M=nb.Jacobi()).solve(nb.AxHelm(), x, _cuda(b),
                                                                       P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert np.abs(_np(x) - xo).max() / np.abs(xo).max() < 1e-7
    # GMRES on the same mesh
    xg = P.zeros()
    mg = nb.GMRES(max_iter=2000, abs_tol=1e-10 * r0, M=nb.Jacobi()).solve(nb.AxHelm(), xg,
                                                                          _cuda(b), P.n, P)
    xgo, it_go, _, _ = O.gmres_jacobi(b, 2000, 1e-10 * r0)
    assert mg.converged and abs(mg.iter - it_go) <= 1, (mg.iter, it_go)


@pytest.mark.parametrize("k,lx", [(36, 4), (60, 5)])
def test_high_valence_vertex_matches_oracle(nb, oracle, k, lx):
    """A point with 8 + k copies, more than a warp has lanes: the gather-
    scatter sums it as a long segment (one thread) beside the warp chunks.
    gs bit-exact without and with the mask (a Jacobi-PCG solve, whose
    operator gather-scatter masks the boundary)."""
    from neko_b200 import workloads
    ids, xyz = workloads.hub_mesh((2, 2, 2), k, rotate_seed=1)
    P = nb.Problem.from_mesh(ids, xyz, lx, deform=0.0, dirichlet=True)
    O = oracle.OracleProblem.from_elements(ids, xyz, lx)
    O.coef()
    O.bc_boundary()
    rng = np.random.default_rng(k)
    u = rng.uniform(-1, 1, P.n)
    g = _cuda(u)
    P.gs.op(g)
    torch.cuda.synchronize()
    assert np.array_equal(_np(g), O.gs_add(u))
    b = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(P.n)))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    xo, it_o, _, _ = O.cg_jacobi(b, 2000, 1e-10 * r0)
    x = P.zeros()
    mon = nb.CG(max_iter=2000, abs_tol=1e-10 * r0, M=nb.Jacobi()).solve(nb.AxHelm(), x, _cuda(b),
                                                                       P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    assert np.abs(_np(x) - xo).max() / np.abs(xo).max() < 1e-7


@pytest.mark.parametrize("nel,lx,seed", [((3, 2, 4), 6, 1), ((3, 3, 3), 8, 2), ((2, 3, 2), 5, 3)])
def test_rotated_mesh_hsmg_matches_oracle(nb, oracle, nel, lx, seed):
    """hsmg on neighbours that meet with arbitrary relative orientation: the
    Schwarz ghost exchange follows each face pairing (the reference reaches
    it through a gather-scatter on the (lx+2)-point numbering).  One apply
    within 1e-10 of the oracle's, flexible CG within +-1 iteration and 1e-7,
    the mixed-precision solve within 1e-6 of the oracle's solution."""
    P, O = _pair(nb, oracle, nel, lx, seed, 0.05)
    rng = np.random.default_rng(seed)
    H = oracle.OracleHsmg(O)
    r = O.bc_apply(O.gs_add(rng.standard_normal(P.n)))
    z = P.zeros()
    nb.Hsmg().solve(z, _cuda(r), P)
    torch.cuda.synchronize()
    zo = H.apply(r)
    assert np.abs(_np(z) - zo).max() <= 1e-10 * np.abs(zo).max()
    b = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(P.n)))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    xo, it_o, _, _ = H.cg(b, 300, 1e-9 * r0, flexible=True)
    for mixed in (False, True):
        x = P.zeros()
        mon = nb.FCG(max_iter=300, abs_tol=1e-9 * r0, M=nb.Hsmg(mixed=mixed)).solve(
            nb.AxHelm(), x, _cuda(b), P.n, P)
        assert mon.converged
        if mixed:
            assert mon.iter <= it_o + 3, (mon.iter, it_o)
            assert np.linalg.norm(_np(x) - xo) / np.linalg.norm(xo) < 1e-6
        else:
            assert abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
            assert np.abs(_np(x) - xo).max() / np.abs(xo).max() < 1e-7


@pytest.mark.parametrize("nel,lx,periodic", [((4, 3, 4), 8, (True,) * 3),
                                             ((3, 4, 3), 6, (False,) * 3)])
def test_unrotated_mesh_solves_like_box(nb, nel, lx, periodic):
    """A box given as an unstructured mesh (no rotation, periodic ids
    merged) solves with hsmg-FCG like the structured box: same iteration
    count, solutions equal to 1e-10."""
    from neko_b200 import workloads
    hi = (2 * np.pi,) * 3 if any(periodic) else (1.0,) * 3
    ids, xyz = workloads.box_mesh(nel, hi=hi, periodic=periodic)
    dirichlet = not all(periodic)
    Pm = nb.Problem.from_mesh(ids, xyz, lx, deform=0.05, dirichlet=dirichlet)
    Pb = nb.Problem(nel, lx, hi=hi, periodic=periodic, deform=0.05, dirichlet=dirichlet)
    assert (Pm.n, Pm.nlocal, Pm.nblocks, Pm.nmask) == (Pb.n, Pb.nlocal, Pb.nblocks, Pb.nmask)
    rng = np.random.default_rng(3)
    f = Pb.zeros()
    f.copy_(_cuda(rng.standard_normal(Pb.n)) * Pb.field("B"))
    if all(periodic):
        f -= f.mean()
    Pb.gs.op(f)
    Pb.bclst.apply(f)
    r0 = float(torch.sqrt((f * Pb.field("mult") * f).sum() / Pb.volume))
    xs = []
    its = []
    for P in (Pb, Pm):
        x = P.zeros()
        mon = nb.FCG(max_iter=200, abs_tol=1e-9 * r0, M=nb.Hsmg()).solve(nb.AxHelm(), x, f.clone(),
                                                                         P.n, P)
        assert mon.converged
        xs.append(_np(x))
        its.append(mon.iter)
    assert its[0] == its[1]
    a, b = xs
    if all(periodic):
        a, b = a - a.mean(), b - b.mean()
    assert np.abs(a - b).max() / np.abs(b).max() < 1e-10


def test_problem_from_nmsh_file(nb, oracle, tmp_path):
    """An .nmsh file in the reference's layout (genmeshbox with periodic
    zones) read by the product and solved with hsmg-FCG: the same iteration
    count and solution (1e-7) as the oracle's box problem."""
    from neko_b200 import workloads
    nel, lx, hi = (4, 4, 3), 6, (2 * np.pi,) * 3
    path = tmp_path / "box.nmsh"
    oracle.genmeshbox_nmsh(path, nel, hi=hi, periodic=(True, True, True))
    ids, xyz = nb.read_nmsh(path)
    P = nb.Problem.from_mesh(ids, xyz, lx, deform=0.05, dirichlet=False)
    O = oracle.OracleProblem.box(nel, lx, hi=hi, periodic=(True,) * 3)
    O.deform_sine(0.05)
    O.coef()
    x, y, z, B = O.f64("x"), O.f64("y"), O.f64("z"), O.f64("B")
    b = O.gs_add(workloads.periodic_box_rhs(x, y, z, B, 4))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    H = oracle.OracleHsmg(O)
    xo, it_o, _, _ = H.cg(b, 200, 1e-8 * r0, flexible=True)
    xd = P.zeros()
    mon = nb.FCG(max_iter=200, abs_tol=1e-8 * r0, M=nb.Hsmg()).solve(nb.AxHelm(), xd, _cuda(b),
                                                                     P.n, P)
    assert mon.converged and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    a = _np(xd)
    a, r = a - a.mean(), xo - xo.mean()
    assert np.abs(a - r).max() / np.abs(r).max() < 1e-7
