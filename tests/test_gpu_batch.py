"""Batched Jacobi-PCG (nb_batch_*): every solve of a heterogeneous batch
equals the same solve run alone through nb_solve, and matches the CPU
oracle's Jacobi-PCG.

Tolerances: iteration counts within +-1 (both are FP64 CG with the same
recurrences; the per-solve sums are formed in a different order);
solutions to 1e-9 relative (rounding amplified by the iteration).
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


def _problem(nb, nel, lx, periodic, deform, h2, seed):
    per = (periodic,) * 3
    P = nb.Problem(nel, lx, hi=(2 * np.pi,) * 3 if periodic else (1.0,) * 3, periodic=per,
                   deform=deform, dirichlet=not periodic)
    rng = np.random.default_rng(seed)
    h1 = torch.full((P.n,), float(rng.uniform(0.5, 2.0)), dtype=torch.float64, device="cuda")
    if h2 is not None:
        P.set_coefficients(h1, torch.full_like(h1, float(h2)))
    else:
        P.set_coefficients(h1)
    f = torch.as_tensor(rng.standard_normal(P.n), device="cuda") * P.field("B")
    if periodic and h2 is None:
        f -= f.mean()
    P.gs.op(f)
    P.bclst.apply(f)
    r0 = float(torch.sqrt((f * P.field("mult") * f).sum() / P.volume))
    return P, f, r0


SPECS = [((2, 2, 2), 4, False, 0.0, 5.0),
         ((3, 2, 4), 6, False, 0.05, 20.0),
         ((4, 4, 4), 8, True, 0.05, 1.0),
         ((2, 3, 2), 10, False, 0.08, None),
         ((5, 5, 5), 6, True, 0.0, 60.0),
         ((6, 4, 3), 8, False, 0.1, 0.0)]


def _alone(nb, P, f, tol, max_iter):
    x = P.zeros()
    mon = nb.CG(max_iter=max_iter, abs_tol=tol, M=nb.Jacobi()).solve(nb.AxHelm(), x, f, P.n, P)
    return x, mon


def test_batch_matches_alone(nb):
    probs = [_problem(nb, *s, seed=i) for i, s in enumerate(SPECS)]
    B = nb.Batch()
    xs, slots = [], []
    for P, f, r0 in probs:
        x = P.zeros()
        xs.append(x)
        slots.append(B.submit(P, f, x, 1e-10 * r0, max_iter=2000))
    assert B.run() == 0
    torch.cuda.synchronize()
    for (P, f, r0), x, s in zip(probs, xs, slots):
        done, mon = B.result(s)
        xa, ma = _alone(nb, P, f, 1e-10 * r0, 2000)
        assert done and mon.converged and ma.converged
        assert abs(mon.iter - ma.iter) <= 1, (P.lx, mon.iter, ma.iter)
        assert abs(mon.res_start - ma.res_start) <= 1e-12 * ma.res_start
        err = float(torch.linalg.norm(x - xa) / torch.linalg.norm(xa))
        assert err < 1e-9, (P.lx, err)
    for lx in (4, 6, 8, 10):
        ks, ms = B.tuning(lx)
        assert ks >= 1 and len(ms) >= 2 and all(m > 0 for m in ms)
    B.close()


def test_batch_matches_oracle(nb, oracle):
    P, f, r0 = _problem(nb, (3, 3, 3), 8, False, 0.05, None, seed=9)
    O = oracle.OracleProblem.box((3, 3, 3), 8, hi=(1.0,) * 3, periodic=(False,) * 3)
    O.deform_sine(0.05)
    O.coef()
    O.bc_boundary()
    h1 = float(P.field("h1")[0])
    O.set_f64("h1", np.full(O.f64("h1").size, h1))
    fo = f.cpu().numpy()
    xo, it_o, rs_o, rf_o = O.cg_jacobi(fo, 1000, 1e-10 * r0)
    B = nb.Batch()
    x = P.zeros()
    s = B.submit(P, f, x, 1e-10 * r0, 1000)
    B.run()
    done, mon = B.result(s)
    assert done and abs(mon.iter - it_o) <= 1, (mon.iter, it_o)
    np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=0, atol=1e-8 * np.abs(xo).max())
    B.close()


def test_batch_budget_admission(nb):
    P, f, r0 = _problem(nb, (4, 4, 4), 8, False, 0.0, 1.0, seed=3)
    need = 4 * P.n * 8
    B = nb.Batch(hbm_budget=int(1.5 * need))
    x1, x2 = P.zeros(), P.zeros()
    s1 = B.submit(P, f, x1, 1e-8 * r0, 500)
    with pytest.raises(nb.NekoB200Error):
        B.submit(P, f, x2, 1e-8 * r0, 500)
    B.release(s1)
    s2 = B.submit(P, f, x2, 1e-8 * r0, 500)  # budget freed
    B.run()
    assert B.result(s2)[0]
    B.close()


def test_continuous_join_equals_alone(nb):
    """Solves that join while others are running end with the same iterates
    as when run alone."""
    probs = [_problem(nb, *s, seed=20 + i) for i, s in enumerate(SPECS[:4])]
    B = nb.Batch()
    xs = [P.zeros() for P, _, _ in probs]
    s0 = B.submit(probs[0][0], probs[0][1], xs[0], 1e-10 * probs[0][2], 2000)
    s1 = B.submit(probs[1][0], probs[1][1], xs[1], 1e-10 * probs[1][2], 2000)
    B.run(max_chunks=2)
    s2 = B.submit(probs[2][0], probs[2][1], xs[2], 1e-10 * probs[2][2], 2000)
    B.run(max_chunks=1)
    s3 = B.submit(probs[3][0], probs[3][1], xs[3], 1e-10 * probs[3][2], 2000)
    B.run()
    for (P, f, r0), x, s in zip(probs, xs, (s0, s1, s2, s3)):
        done, mon = B.result(s)
        xa, ma = _alone(nb, P, f, 1e-10 * r0, 2000)
        assert done and abs(mon.iter - ma.iter) <= 1
        assert float(torch.linalg.norm(x - xa) / torch.linalg.norm(xa)) < 1e-9
    B.close()


def test_batch_rejects_unsupported_lx(nb):
    P = nb.Problem((2, 2, 2), 5)
    B = nb.Batch()
    with pytest.raises(nb.NekoB200Error):
        B.submit(P, P.zeros(), P.zeros(), 1e-8)
    B.close()


def test_scalar_coefficients_share_geometry(nb):
    """Slots with constant coefficients on one shared problem (mesh, G, gs
    maps built once) equal solves on problems whose h1/h2 fields hold the
    same constants."""
    B = nb.Batch()
    shared = nb.Problem((3, 4, 3), 8, deform=0.07)
    rng = np.random.default_rng(17)
    cases = [(1.3, 0.0), (0.6, 45.0), (1.9, 7.5)]
    fs, xs, slots = [], [], []
    for h1, h2 in cases:
        f = torch.as_tensor(rng.standard_normal(shared.n), device="cuda") * shared.field("B")
        shared.gs.op(f)
        shared.bclst.apply(f)
        x = shared.zeros()
        fs.append(f)
        xs.append(x)
        slots.append(B.submit(shared, f, x, 1e-11, 3000, h1=h1, h2=h2))
    B.run()
    for (h1, h2), f, x, s in zip(cases, fs, xs, slots):
        P = nb.Problem((3, 4, 3), 8, deform=0.07)
        c1 = torch.full((P.n,), h1, dtype=torch.float64, device="cuda")
        if h2:
            P.set_coefficients(c1, torch.full_like(c1, h2))
        else:
            P.set_coefficients(c1)
        xa, ma = _alone(nb, P, f, 1e-11, 3000)
        done, mon = B.result(s)
        assert done and mon.converged and abs(mon.iter - ma.iter) <= 1, (mon.iter, ma.iter)
        assert float(torch.linalg.norm(x - xa) / torch.linalg.norm(xa)) < 1e-9
    B.close()
