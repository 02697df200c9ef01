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
