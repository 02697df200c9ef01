"""Served request stream (neko_b200.serve): each request's result is the
same when it runs alone as when it is served in a mix with others that
arrive while it is on the GPU.

The per-solve arithmetic of the batch does not depend on the other slots
(work items, chunks and their summation order are per solve), so with the
same Batch -- hence the same autotuned k-split per lx -- the solutions are
bit-identical and the iteration counts equal.
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


def _small_specs(count, seed):
    from neko_b200 import workloads
    specs = workloads.uneven_specs(count, seed=seed)
    for sp in specs:  # keep the test small: 2..5 elements per side
        sp["n"] = 2 + sp["n"] % 4
    return specs


def test_mix_equals_alone(nb):
    from neko_b200 import serve
    specs = _small_specs(16, seed=5)
    cache = serve.GeometryCache()
    pool = serve.RhsPool(cache)
    B = nb.Batch()
    t_arr = serve.arrivals(2000.0, len(specs), seed=1)  # overlapping arrivals
    lat, it, conv, span, xs = serve.serve_batched(specs, t_arr, pool, 0, batch=B)
    assert all(conv) and all(v is not None and v >= 0 for v in lat)
    for i, sp in enumerate(specs):
        _, it1, conv1, _, xs1 = serve.serve_batched([sp], np.zeros(1), pool, 0, batch=B)
        assert conv1[0] and it1[0] == it[i], (i, it1[0], it[i])
        assert torch.equal(xs1[0], xs[i]), i
    B.close()
    cache.close()


def test_budget_queues_requests(nb):
    """With room for about two solves, every request still completes
    (admission waits for slots to free) with the same results."""
    from neko_b200 import serve
    specs = _small_specs(8, seed=9)
    cache = serve.GeometryCache()
    pool = serve.RhsPool(cache)
    for sp in specs:
        pool.get(sp)
    biggest = max(cache.get(sp).n for sp in specs)
    B = nb.Batch(hbm_budget=int(2.5 * 5 * 8 * biggest))
    lat, it, conv, span, xs = serve.serve_batched(specs, np.zeros(len(specs)), pool, 0, batch=B)
    assert all(conv)
    B2 = nb.Batch()
    lat2, it2, conv2, _, xs2 = serve.serve_batched(specs, np.zeros(len(specs)), pool, 0, batch=B2)
    for i in range(len(specs)):
        assert abs(it[i] - it2[i]) <= 1
        d = float(torch.linalg.norm(xs[i] - xs2[i]) / torch.linalg.norm(xs2[i]))
        assert d < 1e-9
    B.close()
    B2.close()
    cache.close()


def test_sequential_server_agrees(nb):
    from neko_b200 import serve
    specs = _small_specs(6, seed=13)
    cache = serve.GeometryCache()
    pool = serve.RhsPool(cache)
    t_arr = np.zeros(len(specs))
    lat, it, conv, _, _ = serve.serve_batched(specs, t_arr, pool, 0)
    lat_s, it_s, conv_s, _ = serve.serve_sequential(specs, t_arr, pool)
    assert all(conv_s)
    assert max(abs(a - b) for a, b in zip(it, it_s)) <= 1
    cache.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_per_problem_mix_equals_alone(nb, mode):
    """Requests with pc "hsmg" run as per-problem hsmg solves (FP64, or FP32
    smoothing for "mixed") beside batched Jacobi ones; each result is the
    same served alone as in the mix: iteration counts equal, solutions
    bit-identical (every instance of a shape is built the same way and a
    solve's arithmetic does not depend on the others running)."""
    from neko_b200 import serve
    specs = _small_specs(12, seed=21)
    assert {sp["pc"] for sp in specs} == {"jacobi", "hsmg"}
    cache = serve.GeometryCache()
    pool = serve.RhsPool(cache)
    inst = serve.InstancePool(cache, variants=(mode == "mixed",))
    B = nb.Batch()
    t_arr = serve.arrivals(3000.0, len(specs), seed=2)
    lat, it, conv, span, xs = serve.serve_batched(specs, t_arr, pool, 0, batch=B, mode=mode,
                                                  instances=inst, max_solves=4)
    assert all(conv)
    for i, sp in enumerate(specs):
        _, it1, conv1, _, xs1 = serve.serve_batched([sp], np.zeros(1), pool, 0, batch=B,
                                                    mode=mode, instances=inst)
        assert conv1[0] and it1[0] == it[i], (i, it1[0], it[i])
        assert torch.equal(xs1[0], xs[i]), i
    # the per-problem results against the one-by-one FP64 server
    lat_s, it_s, conv_s, _ = serve.serve_sequential(specs, np.zeros(len(specs)), pool,
                                                    mode="fp64")
    assert all(conv_s)
    for i, sp in enumerate(specs):
        if sp["pc"] == "hsmg" and mode == "fp64":
            assert it_s[i] == it[i], (i, it_s[i], it[i])
        else:
            assert abs(it_s[i] - it[i]) <= 3, (i, it_s[i], it[i])
    B.close()
    inst.close()
    cache.close()


def test_submit_solve_equals_nb_solve(nb):
    """A per-problem slot gives bit-for-bit the nb_solve result of the same
    problem and options, here while a batched Jacobi slot runs beside it."""
    from neko_b200 import workloads
    P1 = nb.Problem((4, 4, 4), 8, deform=0.04)
    P2 = nb.Problem((4, 4, 4), 8, deform=0.04)
    Pj = nb.Problem((3, 3, 3), 6, deform=0.02)
    f = workloads.uneven_rhs(P1, 17)
    fj = workloads.uneven_rhs(Pj, 18)
    r0 = float(torch.sqrt((f * P1.field("mult") * f).sum() / P1.volume))
    B = nb.Batch()
    x1, xj = P1.zeros(), Pj.zeros()
    s1 = B.submit_solve(P1, f, x1, 1e-8 * r0, 300, h1=1.3, h2=7.0, pc="hsmg", mixed=True)
    sj = B.submit(Pj, fj, xj, 1e-8, 3000, h1=0.7, h2=2.0)
    B.run()
    d1, m1 = B.result(s1)
    dj, mj = B.result(sj)
    assert d1 and dj and m1.converged and mj.converged
    P2.set_coefficients_const(1.3, 7.0)
    x2 = P2.zeros()
    m2 = nb.FCG(max_iter=300, abs_tol=1e-8 * r0, M=nb.Hsmg(mixed=True)).solve(nb.AxHelm(), x2, f,
                                                                             P2.n, P2)
    torch.cuda.synchronize()
    assert m2.iter == m1.iter and torch.equal(x1, x2)
    B.close()
