"""Entry points used from a caller's non-blocking stream.  Set-up work that
the library does on the legacy stream (workspace clearing, preconditioner
uploads, batch tables) must be complete before the caller's stream reads
it, including on the first call for a fresh problem."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nb():
    import neko_b200
    neko_b200.load()
    return neko_b200


def _rhs(P, seed):
    rng = np.random.default_rng(seed)
    f = torch.as_tensor(rng.standard_normal(P.n), device="cuda") * P.field("B")
    P.gs.op(f)
    P.bclst.apply(f)
    torch.cuda.synchronize()
    return f, math.sqrt(float((f * P.field("mult") * f).sum()) / P.volume)


@pytest.mark.parametrize("pc", ["jacobi", "hsmg"])
def test_first_solve_on_side_stream(nb, pc):
    side = torch.cuda.Stream()
    for k in range(6):
        shape = ((3 + k % 3, 3, 4), (6, 8, 10)[k % 3])
        ref_P = nb.Problem(*shape, deform=0.05)
        P = nb.Problem(*shape, deform=0.05)  # fresh: first solve allocates
        f, r0 = _rhs(ref_P, k)
        M = nb.Jacobi() if pc == "jacobi" else nb.Hsmg()
        Solver = nb.CG if pc == "jacobi" else nb.FCG
        x_ref = ref_P.zeros()
        m_ref = Solver(max_iter=2000, abs_tol=1e-10 * r0, M=M).solve(nb.AxHelm(), x_ref, f,
                                                                     ref_P.n, ref_P)
        with torch.cuda.stream(side):
            x = torch.zeros(P.n, dtype=torch.float64, device="cuda")
            m = Solver(max_iter=2000, abs_tol=1e-10 * r0, M=M).solve(nb.AxHelm(), x, f, P.n, P,
                                                                     stream=side)
        torch.cuda.synchronize()
        assert m.iter == m_ref.iter and m.res_start == m_ref.res_start, (k, m, m_ref)
        assert torch.equal(x, x_ref)


def test_batch_on_side_stream(nb):
    side = torch.cuda.Stream()
    P = nb.Problem((4, 3, 3), 8, deform=0.03)
    f, r0 = _rhs(P, 3)
    B = nb.Batch()
    with torch.cuda.stream(side):
        x = torch.zeros(P.n, dtype=torch.float64, device="cuda")
        s = B.submit(P, f, x, 1e-10 * r0, 2000, h1=1.0, h2=0.0)
        B.run(stream=side)
    torch.cuda.synchronize()
    done, mon = B.result(s)
    Q = nb.Problem((4, 3, 3), 8, deform=0.03)
    xa = Q.zeros()
    ma = nb.CG(max_iter=2000, abs_tol=1e-10 * r0, M=nb.Jacobi()).solve(nb.AxHelm(), xa, f, Q.n, Q)
    assert done and abs(mon.iter - ma.iter) <= 1
    assert float(torch.linalg.norm(x - xa) / torch.linalg.norm(xa)) < 1e-9
    B.close()
