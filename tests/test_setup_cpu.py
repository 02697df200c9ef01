"""Host-side setup of the product library against the oracle (no GPU):
GLL space and the gather-scatter maps must match entry for entry."""
import ctypes

import numpy as np
import pytest


def _nb_gll(nblib, lx):
    z, w, d = (np.zeros(k) for k in (lx, lx, lx * lx))
    P = ctypes.POINTER(ctypes.c_double)
    assert nblib.nb_gll(lx, z.ctypes.data_as(P), w.ctypes.data_as(P), d.ctypes.data_as(P)) == 0
    return z, w, d.reshape(lx, lx, order="F")


@pytest.mark.parametrize("lx", [2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 14, 16])
def test_gll_matches_oracle(nblib, oracle, lx):
    z0, w0, d0 = oracle.gll(lx)
    z1, w1, d1 = _nb_gll(nblib, lx)
    np.testing.assert_allclose(z1, z0, rtol=0, atol=4e-16)
    np.testing.assert_allclose(w1, w0, rtol=1e-14, atol=0)
    np.testing.assert_allclose(d1, d0, rtol=1e-13, atol=1e-13 * np.abs(d0).max())


def nb_maps(nblib, nel, periodic, lx):
    IP = ctypes.POINTER(ctypes.c_int)
    ne = (ctypes.c_int * 3)(*nel)
    pe = (ctypes.c_int * 3)(*[int(p) for p in periodic])
    nl, fo, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    assert nblib.nb_box_gs_maps(ne, pe, lx, ctypes.byref(nl), ctypes.byref(fo), ctypes.byref(nb),
                                None, None, None, None) == 0
    dg = np.zeros(nl.value, np.int32)
    gd = np.zeros(nl.value, np.int32)
    bl = np.zeros(nb.value, np.int32)
    bo = np.zeros(nb.value, np.int32)
    assert nblib.nb_box_gs_maps(ne, pe, lx, ctypes.byref(nl), ctypes.byref(fo), ctypes.byref(nb),
                                dg.ctypes.data_as(IP), gd.ctypes.data_as(IP),
                                bl.ctypes.data_as(IP), bo.ctypes.data_as(IP)) == 0
    return fo.value, dg, gd, bl, bo


CASES = [((2, 2, 2), (0, 0, 0), 3), ((3, 2, 4), (0, 0, 0), 5), ((8, 8, 8), (0, 0, 0), 8),
         ((3, 3, 3), (1, 1, 1), 4), ((4, 3, 5), (1, 0, 1), 6), ((5, 4, 3), (0, 1, 0), 8),
         ((6, 6, 6), (1, 1, 1), 8), ((2, 3, 2), (0, 0, 0), 2), ((3, 3, 4), (1, 1, 1), 10)]


@pytest.mark.parametrize("nel,periodic,lx", CASES)
def test_gs_maps_bit_exact(nblib, oracle, nel, periodic, lx):
    P = oracle.OracleProblem.box(nel, lx, hi=(2 * np.pi,) * 3, periodic=[bool(p) for p in periodic])
    fo, dg, gd, bl, bo = nb_maps(nblib, nel, periodic, lx)
    assert fo == P.local_facet_offset
    np.testing.assert_array_equal(dg, P.i32("dof_gs"))
    np.testing.assert_array_equal(gd, P.i32("gs_dof"))
    np.testing.assert_array_equal(bl, P.i32("blk_len"))
    np.testing.assert_array_equal(bo, P.i32("blk_off"))


def test_periodic_needs_three(nblib):
    IP = ctypes.POINTER(ctypes.c_int)
    ne = (ctypes.c_int * 3)(2, 4, 4)
    pe = (ctypes.c_int * 3)(1, 0, 0)
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = nblib.nb_box_gs_maps(ne, pe, 4, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                              None, None, None, None)
    assert st == 2 and b"at least 3" in nblib.nb_last_error() or b">= 3" in nblib.nb_last_error()


# --- unstructured meshes (nb_mesh_gs_maps) ------------------------------------
def nb_mesh_maps(nblib, ids, lx):
    IP = ctypes.POINTER(ctypes.c_int)
    ids = np.ascontiguousarray(ids, dtype=np.int32)
    nelv = ids.shape[0]
    nl, fo, nb = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    args = (nelv, ids.ctypes.data_as(IP), lx, ctypes.byref(nl), ctypes.byref(fo),
            ctypes.byref(nb))
    assert nblib.nb_mesh_gs_maps(*args, None, None, None, None, None) == 0, \
        nblib.nb_last_error()
    fn = np.zeros(nelv * 6, np.int32)
    dg, gd = np.zeros(nl.value, np.int32), np.zeros(nl.value, np.int32)
    bl, bo = np.zeros(nb.value, np.int32), np.zeros(nb.value, np.int32)
    assert nblib.nb_mesh_gs_maps(*args, *(a.ctypes.data_as(IP) for a in (fn, dg, gd, bl, bo))) == 0
    return fo.value, fn, dg, gd, bl, bo


MESH_CASES = [((3, 2, 4), 5, 1, (False,) * 3), ((4, 4, 4), 6, 2, (False,) * 3),
              ((2, 3, 3), 8, 3, (False,) * 3), ((3, 3, 3), 4, None, (False,) * 3),
              ((3, 4, 3), 6, 5, (True, False, True)), ((3, 3, 3), 7, 6, (True,) * 3)]


@pytest.mark.parametrize("nel,lx,seed,periodic", MESH_CASES)
def test_mesh_gs_maps_bit_exact(nblib, oracle, nel, lx, seed, periodic):
    """Maps of a box meshed as unstructured elements, with every element's
    local frame turned by a random cube rotation (neighbours meet with any
    relative orientation), against the oracle's dofmap + gs_init_mapping."""
    from neko_b200 import workloads
    ids, xyz = workloads.box_mesh(nel, periodic=periodic, rotate_seed=seed)
    P = oracle.OracleProblem.from_elements(ids, xyz, lx)
    fo, fn, dg, gd, bl, bo = nb_mesh_maps(nblib, ids, lx)
    assert fo == P.local_facet_offset
    np.testing.assert_array_equal(dg, P.i32("dof_gs"))
    np.testing.assert_array_equal(gd, P.i32("gs_dof"))
    np.testing.assert_array_equal(bl, P.i32("blk_len"))
    np.testing.assert_array_equal(bo, P.i32("blk_off"))


@pytest.mark.parametrize("k,lx", [(36, 4), (60, 3)])
def test_high_valence_vertex_maps_bit_exact(nblib, oracle, k, lx):
    """A point shared by more elements than a warp has lanes (8 + k copies):
    its gs block is longer than 32 entries."""
    from neko_b200 import workloads
    ids, xyz = workloads.hub_mesh((2, 2, 2), k, rotate_seed=1)
    P = oracle.OracleProblem.from_elements(ids, xyz, lx)
    fo, fn, dg, gd, bl, bo = nb_mesh_maps(nblib, ids, lx)
    assert bl.max() == 8 + k
    assert fo == P.local_facet_offset
    np.testing.assert_array_equal(dg, P.i32("dof_gs"))
    np.testing.assert_array_equal(gd, P.i32("gs_dof"))
    np.testing.assert_array_equal(bl, P.i32("blk_len"))
    np.testing.assert_array_equal(bo, P.i32("blk_off"))


@pytest.mark.parametrize("nel,periodic,lx", CASES[:7])
def test_unrotated_mesh_maps_equal_box_maps(nblib, nel, periodic, lx):
    from neko_b200 import workloads
    ids, _ = workloads.box_mesh(nel, periodic=[bool(p) for p in periodic])
    fo, fn, dg, gd, bl, bo = nb_mesh_maps(nblib, ids, lx)
    fo2, dg2, gd2, bl2, bo2 = nb_maps(nblib, nel, periodic, lx)
    assert fo == fo2
    for a, b in ((dg, dg2), (gd, gd2), (bl, bl2), (bo, bo2)):
        np.testing.assert_array_equal(a, b)


def test_mesh_maps_on_reference_face_fixtures(nblib, oracle):
    """The reference's seven two-element face-orientation meshes."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "gs_face_fixtures.json")) as f:
        fixtures = json.load(f)
    for t in fixtures:
        pts = t["points"]
        ids = np.array([[pts[str(r)]["id"] for r in el] for el in t["elements"]], np.int32)
        xyz = np.array([[pts[str(r)]["xyz"] for r in el] for el in t["elements"]])
        P = oracle.OracleProblem.from_elements(ids, xyz, t["lx"])
        fo, fn, dg, gd, bl, bo = nb_mesh_maps(nblib, ids, t["lx"])
        assert fo == P.local_facet_offset, t["name"]
        np.testing.assert_array_equal(dg, P.i32("dof_gs"))
        np.testing.assert_array_equal(gd, P.i32("gs_dof"))
        assert list(fn) == [0] * 6 + [0] * 6 or fn.max() == 2


def test_mesh_rejects_bad_input(nblib):
    IP = ctypes.POINTER(ctypes.c_int)
    ids = np.array([[1, 2, 3, 4, 5, 6, 7, 7]], np.int32)  # repeated vertex
    a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    st = nblib.nb_mesh_gs_maps(1, ids.ctypes.data_as(IP), 4, ctypes.byref(a), ctypes.byref(b),
                               ctypes.byref(c), None, None, None, None, None)
    assert st == 1 and b"repeats a vertex" in nblib.nb_last_error()


def _read_nmsh(nblib, path):
    IP, DP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    ne = ctypes.c_int()
    assert nblib.nb_mesh_read_nmsh(str(path).encode(), ctypes.byref(ne), None, None, None,
                                   None) == 0, nblib.nb_last_error()
    ids = np.zeros((ne.value, 8), np.int32)
    xyz = np.zeros((ne.value, 8, 3))
    npz, nlz = ctypes.c_int(), ctypes.c_int()
    assert nblib.nb_mesh_read_nmsh(str(path).encode(), ctypes.byref(ne), ids.ctypes.data_as(IP),
                                   xyz.ctypes.data_as(DP), ctypes.byref(npz),
                                   ctypes.byref(nlz)) == 0
    return ids, xyz, npz.value


@pytest.mark.parametrize("nel,periodic,lx", [((3, 2, 4), (0, 0, 0), 5), ((4, 3, 5), (1, 0, 1), 6),
                                             ((3, 3, 3), (1, 1, 1), 4)])
def test_nmsh_read_of_genmeshbox_file(nblib, oracle, tmp_path, nel, periodic, lx):
    """A genmeshbox mesh written in the reference's nmsh layout (periodic
    zones included) and read by the product: the gs maps equal the oracle's
    box maps (the oracle builds them from the same records)."""
    path = tmp_path / "box.nmsh"
    oracle.genmeshbox_nmsh(path, nel, hi=(2.0, 3.0, 1.5), periodic=[bool(p) for p in periodic])
    ids, xyz, npz = _read_nmsh(nblib, path)
    assert npz == 2 * sum(int(p) * nel[(d + 1) % 3] * nel[(d + 2) % 3] for d, p in
                          enumerate(periodic))
    P = oracle.OracleProblem.box(nel, lx, hi=(2.0, 3.0, 1.5), periodic=[bool(p) for p in periodic])
    fo, fn, dg, gd, bl, bo = nb_mesh_maps(nblib, ids, lx)
    assert fo == P.local_facet_offset
    np.testing.assert_array_equal(dg, P.i32("dof_gs"))
    np.testing.assert_array_equal(gd, P.i32("gs_dof"))
    np.testing.assert_array_equal(bl, P.i32("blk_len"))
    np.testing.assert_array_equal(bo, P.i32("blk_off"))
    # element coordinates: the box's grid (x fastest)
    h = np.array([2.0, 3.0, 1.5]) / np.array(nel)
    e = nel[0] * nel[1] * nel[2] - 1
    assert np.allclose(xyz[e, 7], [nel[0] * h[0], nel[1] * h[1], nel[2] * h[2]])


def test_nmsh_write_read_roundtrip(nblib, tmp_path):
    from neko_b200 import workloads
    IP, DP = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    ids, xyz = workloads.box_mesh((3, 2, 2), periodic=(True, False, False), rotate_seed=9)
    path = tmp_path / "m.nmsh"
    assert nblib.nb_mesh_write_nmsh(str(path).encode(), ids.shape[0], ids.ctypes.data_as(IP),
                                    xyz.ctypes.data_as(DP)) == 0
    assert path.stat().st_size == 8 + ids.shape[0] * 228 + 8
    ids2, xyz2, npz = _read_nmsh(nblib, path)
    assert npz == 0
    np.testing.assert_array_equal(ids2, ids)
    np.testing.assert_array_equal(xyz2, xyz)


def test_fld_write_layout(nblib, tmp_path):
    """The fld file layout of fld_file_write (src/io/fld_file.f90:402-560):
    header fields and Fortran e20.13 time, byte-order tag, element ids,
    coordinates per element, the field, then per-element min/max."""
    import struct
    DP = ctypes.POINTER(ctypes.c_double)
    nelv, lx = 3, 4
    l3 = lx ** 3
    rng = np.random.default_rng(2)
    x, y, z, p = (rng.standard_normal(nelv * l3) for _ in range(4))
    path = tmp_path / "field0.f00001"
    assert nblib.nb_fld_write(str(path).encode(), nelv, lx, *(a.ctypes.data_as(DP)
                              for a in (x, y, z, p)), 123.456, 7) == 0
    raw = path.read_bytes()
    hdr = raw[:132].decode()
    assert hdr.startswith("#std 8  4  4  4          3          3  0.1234560000000E+03         7")
    assert hdr.split()[-1] == "XP" and len(hdr) == 132
    assert abs(struct.unpack("<f", raw[132:136])[0] - 6.54321) < 1e-6
    off = 136
    ids = np.frombuffer(raw, np.int32, nelv, off)
    assert list(ids) == [1, 2, 3]
    off += 4 * nelv
    xyz = np.frombuffer(raw, np.float64, 3 * nelv * l3, off).reshape(nelv, 3, l3)
    assert np.array_equal(xyz[:, 0], x.reshape(nelv, l3))
    assert np.array_equal(xyz[:, 2], z.reshape(nelv, l3))
    off += 8 * 3 * nelv * l3
    pp = np.frombuffer(raw, np.float64, nelv * l3, off)
    assert np.array_equal(pp, p)
    off += 8 * nelv * l3
    mx = np.frombuffer(raw, np.float32, 6 * nelv, off).reshape(nelv, 6)
    assert np.allclose(mx[:, 0], x.reshape(nelv, l3).min(1).astype(np.float32))
    assert np.allclose(mx[:, 5], z.reshape(nelv, l3).max(1).astype(np.float32))
    off += 4 * 6 * nelv
    mp = np.frombuffer(raw, np.float32, 2 * nelv, off).reshape(nelv, 2)
    assert np.allclose(mp[:, 1], p.reshape(nelv, l3).max(1).astype(np.float32))
    assert off + 4 * 2 * nelv == len(raw)
