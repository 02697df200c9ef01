"""CPU checks of the ph-multigrid preconditioner (no GPU): the oracle's
restatement (src/multigrid/phmg.f90 with its tree AMG) is a symmetric,
positive operator whose CG beats Jacobi-PCG, its set-up figures are sane,
and the product's host-side aggregation (nb_tamg_aggregate, the same
greedy algorithm in the library) gives the oracle's aggregates on boxes,
periodic boxes, meshes too small for a greedy level and a four-level
hierarchy whose second greedy level runs on aggregate adjacency."""
import numpy as np
import pytest


def _box(oracle, nel, lx, per=(False,) * 3, amp=0.0, hi=1.0, dirichlet=True):
    O = oracle.OracleProblem.box(nel, lx, hi=(hi,) * 3, periodic=per)
    if amp:
        O.deform_sine(amp)
    O.coef()
    if dirichlet:
        O.bc_boundary()
    return O


def test_phmg_setup_figures(oracle):
    O = _box(oracle, (4, 4, 4), 8)
    H = oracle.OraclePhmg(O)
    assert H.levels == 3 and [H.level_lx(i) for i in range(3)] == [8, 4, 2]
    assert H.amg_levels == 3
    assert [H.amg_nodes(i) for i in (1, 2, 3)][0] == 64  # one node an element
    for i in range(2):
        tha, dlt, lam = H.cheby(i)
        # Jacobi-scaled SEM Laplacian: lambda_max of D^-1 A is O(1)
        assert 1.0 < lam < 4.0
        assert tha == pytest.approx((1.1 * lam + lam / 30) / 2)
        assert dlt == pytest.approx((1.1 * lam - lam / 30) / 2)
    for i in range(3):
        assert H.amg_cheby(i)[2] > 0
    H.close()


def test_phmg_apply_symmetric_positive(oracle):
    O = _box(oracle, (3, 4, 3), 6, amp=0.05)
    H = oracle.OraclePhmg(O)
    rng = np.random.default_rng(3)
    mult = O.f64("mult")
    r1, r2 = (O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n))) for _ in range(2))
    z1, z2 = H.apply(r1), H.apply(r2)
    a, b = np.sum(z1 * mult * r2), np.sum(r1 * mult * z2)
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b))
    assert np.sum(z1 * mult * r1) > 0
    # linear: M (r1 + 2 r2) = M r1 + 2 M r2
    z12 = H.apply(r1 + 2 * r2)
    assert np.abs(z12 - (z1 + 2 * z2)).max() <= 1e-10 * np.abs(z12).max()
    H.close()


@pytest.mark.parametrize("kind", ["cg", "fcg", "gmres"])
def test_phmg_krylov_beats_jacobi(oracle, kind):
    O = _box(oracle, (4, 3, 4), 6, amp=0.05)
    H = oracle.OraclePhmg(O)
    rng = np.random.default_rng(5)
    b = O.bc_apply(O.gs_add(O.f64("B") * rng.standard_normal(O.n)))
    r0 = np.sqrt(np.sum(b * O.f64("mult") * b) / O.volume)
    x, it, rs, rf = H.krylov(b, 300, 1e-9 * r0, kind=kind)
    _, it_j, _, _ = O.cg_jacobi(b, 3000, 1e-9 * r0)
    assert rf < 1e-9 * r0 and 0 < it < it_j / 4
    # the residual of the returned solution is the reported one
    w = O.bc_apply(O.gs_add(O.ax_helm(x)))
    res = np.sqrt(np.sum((b - w) * O.f64("mult") * (b - w)) / O.volume)
    assert res == pytest.approx(rf, rel=1e-6, abs=1e-13 * r0)
    H.close()


AGG_CASES = [((4, 4, 4), (False,) * 3, 3),
             ((6, 6, 6), (True,) * 3, 3),
             ((5, 4, 6), (True, False, False), 3),
             ((3, 3, 3), (False,) * 3, 3),      # 27 / 8 < 4: no greedy level
             ((16, 16, 8), (True, True, False), 4)]


@pytest.mark.parametrize("nel,per,levels", AGG_CASES)
def test_product_aggregation_matches_oracle(oracle, nel, per, levels):
    import neko_b200 as nb
    nb.load()
    O = _box(oracle, nel, 4, per=per, dirichlet=not all(per))
    H = oracle.OraclePhmg(O, schedule=(1,), coarse_levels=levels)
    nelv = int(np.prod(nel))
    fn = O.i32("facet_neigh")
    nl, nodes, finest = nb.tamg_aggregate(nelv, 2, fn, levels)
    assert nl == H.amg_levels
    n0 = nelv * 8
    for l in range(1, nl):
        assert nodes[l - 1] == H.amg_nodes(l)
        np.testing.assert_array_equal(finest[l - 1], H.agg_map(l, n0) - 1)
    if nel == (16, 16, 8):
        assert nl == 4 and nodes[2] < nodes[1] < nodes[0]
    H.close()
