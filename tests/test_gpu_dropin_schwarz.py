"""GPU parity of the drop-in tensor / FDM / Schwarz entry points
(cuda_tnsr3d, cuda_fdm_do_fast, cuda_schwarz_extrude, cuda_schwarz_toext3d,
cuda_schwarz_toreg3d) against the oracle's array-level forms of the same
routines.

Tolerances: the index-only routines (toext3d, toreg3d) are bit-exact; the
contractions agree to 1e-13 relative to the largest output (both sides sum
each contraction in ascending index order; only the fused multiply-add
pattern may differ); extrude to 1e-15 relative.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

vp = ctypes.c_void_p


def _cuda(a):
    return torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")


def _ptr(t):
    return vp(t.data_ptr())


def _i(v):
    return ctypes.byref(ctypes.c_int(v))


def _stream():
    return vp(torch.cuda.current_stream().cuda_stream)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("nu,nv", [(8, 4), (4, 8), (4, 2), (2, 4), (10, 4), (5, 7), (16, 16),
                                   (12, 12)])
def test_tnsr3d(oracle, nblib, nu, nv):
    rng = np.random.default_rng(nu * 17 + nv)
    nel = 37
    u = rng.standard_normal(nel * nu ** 3)
    A = rng.standard_normal(nv * nu)
    Bt = rng.standard_normal(nu * nv)
    Ct = rng.standard_normal(nu * nv)
    ref = oracle.tnsr3d(u, nu, nv, A, Bt, Ct, nel)
    v = torch.zeros(nel * nv ** 3, dtype=torch.float64, device="cuda")
    U, dA, dB, dC = _cuda(u), _cuda(A), _cuda(Bt), _cuda(Ct)
    nblib.cuda_tnsr3d(_ptr(v), _i(nv), _ptr(U), _i(nu), _ptr(dA), _ptr(dB), _ptr(dC), _i(nel))
    torch.cuda.synchronize()
    assert _rel(v.cpu().numpy(), ref) < 1e-13


@pytest.mark.parametrize("nl", [4, 6, 7, 8, 10, 12, 16])
def test_fdm_do_fast(oracle, nblib, nl):
    rng = np.random.default_rng(nl)
    nel = 29
    r = rng.standard_normal(nel * nl ** 3)
    s = rng.standard_normal(nel * 6 * nl * nl)
    d = rng.uniform(0.5, 2.0, nel * nl ** 3)
    e_ref, r_ref = oracle.fdm_do_fast(r, s, d, nl, nel)
    E = torch.zeros(nel * nl ** 3, dtype=torch.float64, device="cuda")
    R, S, D = _cuda(r), _cuda(s), _cuda(d)
    nblib.cuda_fdm_do_fast(_ptr(E), _ptr(R), _ptr(S), _ptr(D), _i(nl), _i(nel), _stream())
    torch.cuda.synchronize()
    assert _rel(E.cpu().numpy(), e_ref) < 1e-13
    assert _rel(R.cpu().numpy(), r_ref) < 1e-13  # r is overwritten, as in the reference


@pytest.mark.parametrize("nx,l1,l2,f1,f2,alias", [(6, 0, 2, 1.0, 1.0, True),
                                                  (10, 1, 0, 0.0, 1.0, False),
                                                  (10, 0, 2, 1.0, -1.0, True),
                                                  (3, 0, 1, 0.5, 2.0, False)])
def test_schwarz_extrude(oracle, nblib, nx, l1, l2, f1, f2, alias):
    rng = np.random.default_rng(nx + l1)
    nel = 23
    a1 = rng.standard_normal(nel * nx ** 3)
    a2 = a1 if alias else rng.standard_normal(nel * nx ** 3)
    ref = oracle.schwarz_extrude(a1, l1, f1, a2, l2, f2, nx, nel)
    A1 = _cuda(a1)
    A2 = A1 if alias else _cuda(a2)
    c1, c2 = ctypes.c_double(f1), ctypes.c_double(f2)
    nblib.cuda_schwarz_extrude(_ptr(A1), _i(l1), ctypes.byref(c1), _ptr(A2), _i(l2),
                               ctypes.byref(c2), _i(nx), _i(nel), _stream())
    torch.cuda.synchronize()
    assert _rel(A1.cpu().numpy(), ref) < 1e-15


@pytest.mark.parametrize("nx", [2, 4, 8, 14])
def test_schwarz_toext_toreg(oracle, nblib, nx):
    rng = np.random.default_rng(nx)
    nel = 31
    b = rng.standard_normal(nel * nx ** 3)
    ref_a = oracle.schwarz_toext3d(b, nx, nel)
    B = _cuda(b)
    A = torch.full((nel * (nx + 2) ** 3,), 7.0, dtype=torch.float64, device="cuda")
    nblib.cuda_schwarz_toext3d(_ptr(A), _ptr(B), _i(nx), _i(nel), _stream())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(A.cpu().numpy(), ref_a)
    B2 = torch.zeros_like(B)
    nblib.cuda_schwarz_toreg3d(_ptr(B2), _ptr(A), _i(nx), _i(nel), _stream())
    torch.cuda.synchronize()
    np.testing.assert_array_equal(B2.cpu().numpy(), oracle.schwarz_toreg3d(ref_a, nx, nel))
    np.testing.assert_array_equal(B2.cpu().numpy(), b)
