"""A solver workspace keeps one captured iteration graph and reads each
solve's x and f through its device state, so consecutive solves into
different buffers must give exactly the results of solves on a fresh
problem (the graph follows the new buffers, nothing of the previous solve
leaks in).  Covers CG (Jacobi; hsmg flexible, FP64 and mixed with its
scheduled true residual), restarted GMRES, pipelined CG and the coupled
three-component CG."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import neko_b200
    neko_b200.load()
    return neko_b200


def _problem(nb):
    return nb.Problem((3, 3, 3), 6, deform=0.05, dirichlet=True)


def _rhs(nb, P, seed):
    rng = np.random.default_rng(seed)
    f = torch.as_tensor(rng.standard_normal(P.n), device="cuda") * P.field("B")
    P.gs.op(f)
    P.bclst.apply(f)
    return f


def _solvers(nb):
    return {
        "cg_jacobi": lambda: nb.CG(max_iter=500, abs_tol=1e-9, M=nb.Jacobi()),
        "fcg_hsmg": lambda: nb.FCG(max_iter=200, abs_tol=1e-9, M=nb.Hsmg()),
        "fcg_hsmg_mixed": lambda: nb.FCG(max_iter=200, abs_tol=1e-9, M=nb.Hsmg(mixed=True)),
        "gmres_jacobi": lambda: nb.GMRES(max_iter=500, abs_tol=1e-9, M=nb.Jacobi(), m_restart=20),
        "pipecg_jacobi": lambda: nb.PipeCG(max_iter=500, abs_tol=1e-9, M=nb.Jacobi()),
    }


@pytest.mark.parametrize("name", ["cg_jacobi", "fcg_hsmg", "fcg_hsmg_mixed", "gmres_jacobi",
                                  "pipecg_jacobi"])
def test_new_buffers_reuse_the_graph(nb, name):
    make = _solvers(nb)[name]
    P = _problem(nb)
    outs = []
    for seed in (1, 2, 3):  # a new x and f every solve
        f = _rhs(nb, P, seed)
        x = P.zeros()
        mon = make().solve(nb.AxHelm(), x, f, P.n, P)
        torch.cuda.synchronize()
        outs.append((x.cpu().numpy(), mon.iter, f))
    for seed, (x, it, f) in zip((1, 2, 3), outs):
        Q = _problem(nb)  # fresh problem: a fresh workspace and graph
        fq = f.clone()
        xq = Q.zeros()
        mq = make().solve(nb.AxHelm(), xq, fq, Q.n, Q)
        torch.cuda.synchronize()
        assert mq.iter == it, (name, seed)
        np.testing.assert_array_equal(x, xq.cpu().numpy())
        Q.close()
    P.close()


def test_coupled_new_buffers_reuse_the_graph(nb):
    P = _problem(nb)
    res = []
    for seed in (4, 5):
        f = [_rhs(nb, P, seed + 10 * c) for c in range(3)]
        xs = [P.zeros() for _ in range(3)]
        mons = nb.CoupledCG(max_iter=800, abs_tol=1e-9, M=nb.Jacobi()).solve_coupled(
            nb.AxHelmFull(), *xs, *f, P.n, P)
        torch.cuda.synchronize()
        res.append(([x.cpu().numpy() for x in xs], mons[0].iter, f))
    for xs, it, f in res:
        Q = _problem(nb)
        xq = [Q.zeros() for _ in range(3)]
        mq = nb.CoupledCG(max_iter=800, abs_tol=1e-9, M=nb.Jacobi()).solve_coupled(
            nb.AxHelmFull(), *xq, *[a.clone() for a in f], Q.n, Q)
        torch.cuda.synchronize()
        assert mq[0].iter == it
        for a, b in zip(xs, xq):
            np.testing.assert_array_equal(a, b.cpu().numpy())
        Q.close()
    P.close()
