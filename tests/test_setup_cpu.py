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
