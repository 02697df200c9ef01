"""The velocity solve's full-stress operator and coupled CG against the
oracle's restatements: ax_helm_stress_lx (src/math/bcknd/cpu/
ax_helm_full_cpu.f90:181-375, plus the h2 B term of :164-176) and
cg_cpld_device_solve (src/krylov/bcknd/device/cg_cpld_device.f90:292-417).

Bars: cofactors and 1/jac 1e-12 of their scale; the operator 1e-12 relative
(max-norm) for lx <= 10, 1e-11 above (derivative entries grow like lx^2);
coupled-CG iteration counts within +-1 with Jacobi (10 % without a
preconditioner) and solutions within 1e-7 relative.
Orders 4, 6 and 8 run the streaming kernel, the others the general one
(13 the register-flux form)."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

COF = ("drdx", "drdy", "drdz", "dsdx", "dsdy", "dsdz", "dtdx", "dtdy", "dtdz", "jacinv")


@pytest.fixture(scope="module")
def nb():
    import neko_b200
    neko_b200.load()
    return neko_b200


def _np(t):
    return t.detach().cpu().numpy()


def _cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a), device="cuda")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _rtol(lx):
    return 1e-12 if lx <= 10 else 1e-11


def _pair(nb, oracle, nel, lx, periodic=(False,) * 3, deform=0.05, hi=1.0, dirichlet=True):
    P = nb.Problem(nel, lx, hi=(hi,) * 3, periodic=periodic, deform=deform, dirichlet=dirichlet)
    O = oracle.OracleProblem.box(nel, lx, hi=(hi,) * 3, periodic=periodic)
    if deform:
        O.deform_sine(deform)
    O.coef()
    if dirichlet:
        O.bc_boundary()
    return P, O


def _set_h(P, O, rng, ifh2):
    h1 = rng.uniform(0.5, 2.0, P.n)
    O.set_f64("h1", h1)
    if ifh2:
        h2 = rng.uniform(0.0, 50.0, P.n)
        P.set_coefficients(_cuda(h1), _cuda(h2))
        O.set_f64("h2", h2)
        O.set_ifh2(True)
    else:
        P.set_coefficients(_cuda(h1))


def test_cofactors_match_oracle(nb, oracle):
    """Cofactors to 1e-12 of the scale of the diagonal ones (the cross terms
    are small on a mildly deformed box, so they are measured on that scale,
    as the G factors are); 1/jac to 1e-12 of its own scale."""
    P, O = _pair(nb, oracle, (3, 2, 4), 7)
    scale = max(np.abs(O.f64(k)).max() for k in ("drdx", "dsdy", "dtdz"))
    for name in COF:
        a, b = _np(P.field(name)), O.f64(name)
        sc = np.abs(b).max() if name == "jacinv" else scale
        assert np.abs(a - b).max() <= 1e-12 * sc, name


@pytest.mark.parametrize("lx,ifh2", [(2, False), (3, True), (4, False), (5, True), (6, False),
                                     (6, True), (8, False), (8, True), (10, True), (12, False),
                                     (13, True)])
def test_ax_stress_matches_oracle(nb, oracle, lx, ifh2):
    nel = (3, 2, 3) if lx <= 8 else (3, 2, 2)
    P, O = _pair(nb, oracle, nel, lx, periodic=(True, False, False), hi=2 * np.pi)
    rng = np.random.default_rng(lx)
    _set_h(P, O, rng, ifh2)
    u, v, w = (rng.uniform(-1, 1, P.n) for _ in range(3))
    out = [P.zeros() for _ in range(3)]
    nb.AxHelmFull().compute_vector(*out, _cuda(u), _cuda(v), _cuda(w), P)
    torch.cuda.synchronize()
    ref = O.ax_helm_stress(u, v, w)
    for c in range(3):
        assert _rel(_np(out[c]), ref[c]) <= _rtol(lx), (c, _rel(_np(out[c]), ref[c]))


def test_ax_stress_rigid_motions_in_kernel(nb, oracle):
    """Translations and rotations have zero strain: A_stress of them is
    rounding noise against the operator's scale."""
    P, _ = _pair(nb, oracle, (4, 3, 3), 8, deform=0.05)
    x, y, z = P.field("x"), P.field("y"), P.field("z")
    out = [P.zeros() for _ in range(3)]
    one, zero = torch.ones_like(x), torch.zeros_like(x)
    rng = np.random.default_rng(1)
    rnd = [_cuda(rng.uniform(-1, 1, P.n)) for _ in range(3)]
    nb.AxHelmFull().compute_vector(*out, *rnd, P)
    scale = max(float(o.abs().max()) for o in out)
    for field in ((one, zero, zero), (zero, one, zero), (-y, x, zero), (zero, -z, y)):
        nb.AxHelmFull().compute_vector(*out, *field, P)
        torch.cuda.synchronize()
        assert max(float(o.abs().max()) for o in out) < 1e-11 * scale


def test_drop_in_stress_vector(nb, oracle, nblib):
    """cuda_ax_helm_stress_vector and _part2 with the reference's argument
    lists, dx, dy and dz passed as separate arrays (as Neko's space_t holds
    them)."""
    lx = 8
    P, O = _pair(nb, oracle, (3, 3, 3), lx, periodic=(True,) * 3, hi=2 * np.pi,
                 dirichlet=False)
    rng = np.random.default_rng(21)
    _set_h(P, O, rng, True)
    u, v, w = (rng.uniform(-1, 1, P.n) for _ in range(3))
    ud, vd, wd = _cuda(u), _cuda(v), _cuda(w)
    out = [P.zeros() for _ in range(3)]
    dx = P.field("dx")
    dy, dz = dx.clone(), dx.clone()
    dxt = P.field("dxt")
    w3 = _cuda(O.f64("w3"))
    cof = {k: P.field(k) for k in COF}
    vp = lambda t: ctypes.c_void_p(t.data_ptr())
    nelv, lxc, n = ctypes.c_int(P.nelv), ctypes.c_int(lx), ctypes.c_int(P.n)
    nblib.cuda_ax_helm_stress_vector(*(vp(t) for t in out), vp(ud), vp(vd), vp(wd), vp(dx),
                                     vp(dy), vp(dz), vp(dxt), vp(dxt), vp(dxt),
                                     vp(P.field("h1")), *(vp(cof[k]) for k in COF[:9]),
                                     vp(cof["jacinv"]), vp(w3), ctypes.byref(nelv),
                                     ctypes.byref(lxc))
    nblib.cuda_ax_helm_stress_vector_part2(*(vp(t) for t in out), vp(ud), vp(vd), vp(wd),
                                           vp(P.field("h2")), vp(P.field("B")), ctypes.byref(n))
    torch.cuda.synchronize()
    ref = O.ax_helm_stress(u, v, w)
    for c in range(3):
        assert _rel(_np(out[c]), ref[c]) <= 1e-12


def _rhs(O, rng):
    return [O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n))) for _ in range(3)]


@pytest.mark.parametrize("stress,jacobi,lx", [(True, True, 6), (True, True, 8), (True, False, 5),
                                              (False, True, 8), (True, True, 10)])
def test_coupled_cg_matches_oracle(nb, oracle, stress, jacobi, lx):
    nel = (3, 3, 2) if lx <= 8 else (2, 2, 2)
    P, O = _pair(nb, oracle, nel, lx, deform=0.05)
    rng = np.random.default_rng(100 + lx)
    _set_h(P, O, rng, True)  # a velocity-type solve: h1 = viscosity, h2 = density / dt
    f = _rhs(O, rng)
    r0 = np.sqrt(sum(np.sum(a * O.f64("mult") * a) for a in f) / O.volume)
    tol = 1e-10 * r0
    xo, it_o, _, _ = O.cg_coupled(f, 3000, tol, stress=stress, jacobi=jacobi)
    xs = [P.zeros() for _ in range(3)]
    Ax = nb.AxHelmFull() if stress else nb.AxHelm()
    mons = nb.CoupledCG(max_iter=3000, abs_tol=tol, M=nb.Jacobi() if jacobi else None
                        ).solve_coupled(Ax, *xs, *(_cuda(a) for a in f), P.n, P)
    assert mons[0].converged
    # Jacobi: +-1.  Unpreconditioned CG over 100+ iterations loses
    # orthogonality at a rate set by rounding (the operator's and the
    # reductions' orders differ from the oracle's), so its count is held to
    # 10 % instead.
    slack = 1 if jacobi else max(1, it_o // 10)
    assert abs(mons[0].iter - it_o) <= slack, (mons[0].iter, it_o)
    for c in range(3):
        assert _rel(_np(xs[c]), xo[c]) < 1e-7, c


def test_coupled_cg_refuses_hsmg_and_single_field(nb, oracle):
    P, _ = _pair(nb, oracle, (2, 2, 2), 5)
    f = [P.zeros() for _ in range(3)]
    with pytest.raises(nb.NekoB200Error) as ei:
        nb.CoupledCG(M=nb.Hsmg()).solve_coupled(nb.AxHelmFull(), *[P.zeros() for _ in range(3)],
                                                *f, P.n, P)
    assert ei.value.status == 2
    with pytest.raises(nb.NekoB200Error):
        nb.CoupledCG().solve(nb.AxHelmFull(), P.zeros(), f[0], P.n, P)
    with pytest.raises(nb.NekoB200Error):
        nb.AxHelmFull().compute(P.zeros(), f[0], P)
