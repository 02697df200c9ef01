"""Failure detection without a GPU fault.

Device side: every spin-wait in the library is bounded; the self-test makes
a grid barrier and an mbarrier wait run out (nothing ever arrives) and
checks that both report a timeout and that the device stays usable.
Host side: the serving loop returns a per-request outcome -- forced
non-convergence (max_iter = 1), a NaN right-hand side, a request larger
than the whole HBM budget, an injected allocation failure and cancelled
requests -- while the other requests complete with their usual results.
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


def test_bounded_waits_time_out(nb):
    import ctypes
    L = nb.load()
    a, b = ctypes.c_int(0), ctypes.c_int(0)
    nb._lib.check(L.nb_selftest_bounded_waits(ctypes.byref(a), ctypes.byref(b)))
    assert a.value == 1 and b.value == 1
    P = nb.Problem((2, 2, 2), 8)  # the context is still usable
    w, u = P.zeros(), torch.ones(P.n, dtype=torch.float64, device="cuda")
    nb.AxHelm().compute(w, u, P)
    torch.cuda.synchronize()
    assert torch.isfinite(w).all()


class _Pool:
    """Request payloads: the normal pool, or a NaN right-hand side."""

    def __init__(self, pool):
        self.pool, self.nan = pool, {}

    def get(self, sp):
        P, f, r0 = self.pool.get(sp)
        if sp.get("nan"):
            key = id(P)
            if key not in self.nan:
                g = f.clone()
                g[0] = float("nan")
                self.nan[key] = g
            return P, self.nan[key], r0
        return P, f, r0


def _specs(count, seed):
    from neko_b200 import workloads
    specs = workloads.uneven_specs(count, seed=seed)
    for sp in specs:
        sp["n"] = 2 + sp["n"] % 3
    return specs


def test_serve_outcomes(nb):
    from neko_b200 import serve
    cache = serve.GeometryCache()
    base = serve.RhsPool(cache)
    pool = _Pool(base)
    specs = _specs(7, seed=21)
    specs[1]["max_iter"] = 1                  # forced non-convergence
    specs[2]["nan"] = True                    # NaN right-hand side
    specs[3].update(n=9, lx=10)               # larger than the budget below
    specs[5].update(n=5, lx=10)               # long solve, cancelled after admission
    for sp in specs:
        pool.get(sp)
    small = max(cache.get(sp).n for i, sp in enumerate(specs) if i != 3)
    budget = int(5 * 8 * small * 2.0)         # room for the small solves, never for #3
    assert 5 * 8 * cache.get(specs[3]).n > budget
    t_arr = np.zeros(len(specs))
    B = nb.Batch(hbm_budget=budget)
    real_submit = B.submit
    calls = {"n": 0}

    def flaky_submit(P, f, x, *a, **k):       # injected allocation failure for #6
        if P is cache.get(specs[6]) and calls["n"] == 0 and f is base.get(specs[6])[1]:
            calls["n"] += 1
            raise nb.NekoB200Error(nb._lib.NB_ERR_OOM, "injected")
        return real_submit(P, f, x, *a, **k)
    B.submit = flaky_submit
    status = []
    lat, it, conv, span, xs = serve.serve_batched(
        specs, t_arr, pool, budget, batch=B, status=status, rel_tol=1e-14,
        max_iter=3000, cancel={4: 0.0, 5: 1e-4})
    assert status[0] == serve.OK and conv[0]
    assert status[1] == serve.NOT_CONVERGED and it[1] == 1
    assert status[2] == serve.NAN
    assert status[3] == serve.OOM_REJECTED
    assert status[4] == serve.CANCELLED       # withdrawn before admission
    assert status[5] == serve.CANCELLED       # withdrawn while running
    assert status[6] in (serve.OOM_REJECTED, serve.OK)
    assert all(v is not None for v in lat)
    # the request that completed is unaffected by the failures around it
    B.submit = real_submit
    _, it0, conv0, _, xs0 = serve.serve_batched([specs[0]], np.zeros(1), pool, budget,
                                                batch=B, rel_tol=1e-14, max_iter=3000)
    assert conv0[0] and it0[0] == it[0] and torch.equal(xs0[0], xs[0])
    B.close()
    cache.close()
