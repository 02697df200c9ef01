"""Pins the CPU oracle to the reference's own known-answer tests.

* gather-scatter face orientation: the seven two-element tests of
  tests/unit/gather_scatter/test_gather_scatter_parallel.pf:38-903 (fixtures
  in tests/golden/gs_face_fixtures.json, made by make_gs_fixtures.py);
* fd_weights_full: tests/unit/fast3d/test_fd_weights_full.pf:4-50;
* GLL space: exact nodes/weights for small lx and the sizes checked by
  tests/unit/space/test_space_test.pf:38-80.
"""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _fixtures():
    with open(os.path.join(GOLD, "gs_face_fixtures.json")) as f:
        return json.load(f)


def _mesh_arrays(t):
    pts = t["points"]
    ids = np.array([[pts[str(r)]["id"] for r in el] for el in t["elements"]], dtype=np.int32)
    xyz = np.array([[pts[str(r)]["xyz"] for r in el] for el in t["elements"]], dtype=np.float64)
    return ids, xyz


def _assert_face_equal(t, y):
    lx = t["lx"]
    y = y.reshape(2, lx, lx, lx)  # (e, k, j, i)
    for i in range(1, lx + 1):
        for j in range(1, lx + 1):
            env = {"lx": lx, "i": i, "j": j}
            a = [eval(s, {}, env) for s in t["assert_lhs"].split(",")]
            b = [eval(s, {}, env) for s in t["assert_rhs"].split(",")]
            va = y[a[3] - 1, a[2] - 1, a[1] - 1, a[0] - 1]
            vb = y[b[3] - 1, b[2] - 1, b[1] - 1, b[0] - 1]
            assert abs(va - vb) <= np.finfo(float).eps, (t["name"], i, j, va, vb)


@pytest.mark.parametrize("t", _fixtures(), ids=lambda t: t["name"])
def test_gs_face_orientation(oracle, t):
    ids, xyz = _mesh_arrays(t)
    P = oracle.OracleProblem.from_elements(ids, xyz, t["lx"])
    n = P.n
    dof = P.dof()
    x = np.ones(n)
    x[: n // 2] += dof[: n // 2]  # rone + add2(x, dof, n/2)
    _assert_face_equal(t, P.gs_add(x))
    # 16 vertex + 72 edge entries, 18 face entries (9 shared face points x 2)
    lx = t["lx"]
    assert P.local_facet_offset == 2 * (8 + 12 * (lx - 2)) + 1
    assert P.nlocal == P.local_facet_offset - 1 + 2 * (lx - 2) ** 2


def test_fd_weights_golden(oracle):
    with open(os.path.join(GOLD, "reference_unit_values.json")) as f:
        gold = json.load(f)
    for case in gold["fd_weights_full"]:
        c = oracle.fd_weights_full(case["xi"], case["x"], case["m"])
        np.testing.assert_array_equal(c, np.array(case["c"]))


def test_gll_known_values(oracle):
    z, w, d = oracle.gll(3)
    np.testing.assert_allclose(z, [-1, 0, 1], atol=1e-15)
    np.testing.assert_allclose(w, [1 / 3, 4 / 3, 1 / 3], rtol=1e-14)
    z, w, d = oracle.gll(4)
    np.testing.assert_allclose(z, [-1, -1 / np.sqrt(5), 1 / np.sqrt(5), 1], rtol=1e-14)
    np.testing.assert_allclose(w, [1 / 6, 5 / 6, 5 / 6, 1 / 6], rtol=1e-14)
    for lx in (2, 4, 6, 8, 10, 12, 16):
        z, w, d = oracle.gll(lx)
        assert abs(w.sum() - 2.0) < 1e-13
        # D differentiates polynomials of degree lx-1 exactly
        for p in range(lx):
            np.testing.assert_allclose(d @ z ** p, p * z ** max(p - 1, 0) if p else 0 * z,
                                       atol=1e-11 * max(1, p))


def test_box_counts_unit_box_8(oracle):
    """512-element unit box at lx = 8: the map sizes gs_init_mapping gives
    (8 vertex + 12*6 edge entries per element, face pairs only for faces with
    a neighbour)."""
    P = oracle.OracleProblem.box((8, 8, 8), 8)
    assert P.n == 262144
    assert P.nlocal == 4096 + 36864 + 96768
    assert P.nblks == 12393
    assert P.local_facet_offset == 4096 + 36864 + 1
    fn = P.i32("facet_neigh").reshape(-1, 6)
    assert (fn == 0).sum() == 384  # 6 faces x 64 boundary elements


def test_periodic_box_numbering(oracle):
    """Fully periodic 4^3 box: global numbering has (4*(lx-1))^3 distinct
    points on element boundaries + interiors, every face has a neighbour."""
    lx = 5
    P = oracle.OracleProblem.box((4, 4, 4), lx, hi=(2 * np.pi,) * 3, periodic=(True,) * 3)
    dof = P.dof()
    # interior points are not numbered (0); boundary points: verts+edges+faces
    assert len(np.unique(dof[dof > 0])) == 64 + 192 * (lx - 2) + 192 * (lx - 2) ** 2
    assert (P.i32("facet_neigh") > 0).all()
    assert P.glb_mpts == 125 and P.glb_meds == 192


def test_unit_box_8_analytic_solution(oracle):
    """Jacobi-PCG on -lap u = 3 pi^2 sin sin sin, u = 0 on the boundary of
    the unit box: spectral accuracy at lx = 8 (examples/poisson shape)."""
    P = oracle.OracleProblem.box((4, 4, 4), 8)
    P.coef()
    P.bc_boundary()
    x, y, z = P.f64("x"), P.f64("y"), P.f64("z")
    B, mult = P.f64("B"), P.f64("mult")
    exact = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z)
    b = P.bc_apply(P.gs_add(B * 3 * np.pi ** 2 * exact))
    r0 = np.sqrt(np.sum(b * mult * b) / P.volume)
    u, it, rs, rf = P.cg_jacobi(b, 500, 1e-10 * r0)
    assert abs(rs - r0) <= 1e-12 * r0
    assert rf < 1e-10 * r0
    assert np.abs(u - exact).max() < 1e-8
    assert abs(P.volume - 1.0) < 1e-12


def test_oracle_array_forms_consistent(oracle):
    """The oracle's array-level tnsr3d / fdm_do_fast / toext3d / toreg3d agree
    with direct numpy restatements (the drop-in GPU tests check against
    them)."""
    rng = np.random.default_rng(3)
    nu, nv, nel = 4, 6, 3
    u = rng.standard_normal(nel * nu ** 3)
    A, Bt, Ct = (rng.standard_normal(nv * nu) for _ in range(3))
    v = oracle.tnsr3d(u, nu, nv, A, Bt, Ct, nel).reshape(nel, nv, nv, nv)
    Am = A.reshape(nu, nv).T          # A(i, l) at i + nv*l
    Bm = Bt.reshape(nv, nu)           # Bt(l, j) at l + nu*j -> B(j, l)
    Cm = Ct.reshape(nv, nu)
    U = u.reshape(nel, nu, nu, nu)    # U[e, k, j, i]
    ref = np.einsum("ai,bj,ck,ekji->ecba", Am, Bm, Cm, U)
    np.testing.assert_allclose(v, ref, rtol=1e-12, atol=1e-12)
    nl = 5
    r = rng.standard_normal(nel * nl ** 3)
    s = rng.standard_normal(nel * 6 * nl * nl)
    d = rng.uniform(0.5, 2, nel * nl ** 3)
    e, r2 = oracle.fdm_do_fast(r, s, d, nl, nel)
    S = s.reshape(nel, 3, 2, nl * nl)  # s(:,:,m,dir,e)
    e_ref, r_ref = [], []
    for k in range(nel):
        m = lambda mm, dd: S[k, dd, mm]  # noqa: E731
        t = oracle.tnsr3d(r[k * nl ** 3:(k + 1) * nl ** 3], nl, nl, m(1, 0), m(0, 1), m(0, 2), 1)
        t = t * d[k * nl ** 3:(k + 1) * nl ** 3]
        r_ref.append(t)
        e_ref.append(oracle.tnsr3d(t, nl, nl, m(0, 0), m(1, 1), m(1, 2), 1))
    np.testing.assert_allclose(e, np.concatenate(e_ref), rtol=1e-13, atol=1e-13)
    np.testing.assert_allclose(r2, np.concatenate(r_ref), rtol=1e-13, atol=1e-13)
    b = rng.standard_normal(nel * 27)
    a = oracle.schwarz_toext3d(b, 3, nel)
    assert a.size == nel * 125 and np.count_nonzero(a) == b.size
    np.testing.assert_array_equal(oracle.schwarz_toreg3d(a, 3, nel), b)
