"""Part-1 drop-ins as a linked Neko build uses them.

* Streams: the entry points that take no stream (cuda_ax_helm, cuda_tnsr3d,
  cuda_jacobi_update, the fused-CG helpers) must launch on Neko's
  non-blocking `glb_cmd_queue`, as the reference's kernels do
  (src/math/bcknd/device/cuda/ax_helm.cu:77).  A small shared library that
  defines `glb_cmd_queue` stands in for the Neko executable; a slow producer
  writes the operator's input on that stream and cuda_ax_helm is called
  without any device synchronisation.
* The vector drop-ins not covered elsewhere (copy, rzero, col2, addcol3,
  radd, glsum, glsc2), the device `ortho` built from glsum and radd
  (src/math/operators.f90:349-368), and the fused-CG helpers
  (src/krylov/bcknd/device/cuda/fusedcg_aux.cu:61-87) against numpy.
* The per-problem error word of the streaming kernels: a timeout recorded
  on one problem is reported by that problem only, once.
"""
import ctypes
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
vp = ctypes.c_void_p


def _ptr(t):
    return vp(t.data_ptr())


def _stream():
    return vp(torch.cuda.current_stream().cuda_stream)


def _close(got, ref):
    """Element-wise updates of the form a + b c: the device may fuse them
    into one multiply-add (as the reference's kernels, built with nvcc's
    default contraction, do), so they agree with numpy to a rounding."""
    assert np.abs(got - ref).max() <= 4e-15 * max(np.abs(ref).max(), 1.0)


QUEUE_CHILD = textwrap.dedent(r"""
    import ctypes, sys
    import numpy as np
    import torch
    sys.path.insert(0, sys.argv[2])
    stub = ctypes.CDLL(sys.argv[1], mode=ctypes.RTLD_GLOBAL)   # defines glb_cmd_queue
    import neko_b200 as nb
    from neko_b200 import _lib
    from oracle import oracle
    L = _lib.load()
    torch.cuda.set_device(0)
    nel, lx = (4, 4, 4), 8
    P = nb.Problem(nel, lx, deform=0.05)
    O = oracle.OracleProblem.box(nel, lx)
    O.deform_sine(0.05)
    O.coef()
    rng = np.random.default_rng(3)
    u_host = rng.uniform(-1, 1, P.n)
    ref = O.ax_helm(u_host)
    queue = torch.cuda.Stream()              # created non-blocking by torch
    u_src = torch.as_tensor(u_host, device="cuda")
    u = torch.zeros(P.n, dtype=torch.float64, device="cuda")
    w = torch.zeros(P.n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ctypes.c_void_p.in_dll(stub, "glb_cmd_queue").value = queue.cuda_stream
    f = {k: P.field(k) for k in ("dx", "dxt", "h1", "g11", "g22", "g33", "g12", "g13", "g23")}
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    with torch.cuda.stream(queue):
        torch.cuda._sleep(400_000_000)       # slow producer, then u is written
        u.copy_(u_src)
    # no synchronisation: only the stream order makes u ready for the operator
    L.cuda_ax_helm(p(w), p(u), p(f["dx"]), p(f["dx"]), p(f["dx"]), p(f["dxt"]), p(f["dxt"]),
                   p(f["dxt"]), p(f["h1"]), p(f["g11"]), p(f["g22"]), p(f["g33"]), p(f["g12"]),
                   p(f["g13"]), p(f["g23"]), ctypes.byref(ctypes.c_int(P.nelv)),
                   ctypes.byref(ctypes.c_int(lx)))
    with torch.cuda.stream(queue):
        got = w.cpu().numpy()                # read back in the queue's order
    err = np.abs(got - ref).max() / np.abs(ref).max()
    print("ERR", err)
    assert err < 1e-12, err
""")


def test_dropin_ax_helm_runs_on_glb_cmd_queue(tmp_path):
    stub_c = tmp_path / "neko_queue_stub.c"
    stub_c.write_text("void *glb_cmd_queue = 0;\n")
    stub_so = tmp_path / "libneko_queue_stub.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-o", str(stub_so), str(stub_c)], check=True)
    child = tmp_path / "child.py"
    child.write_text(QUEUE_CHILD)
    r = subprocess.run([sys.executable, str(child), str(stub_so), ROOT], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "ERR" in r.stdout


def test_set_default_stream_orders_tnsr3d(oracle, nblib):
    """nb_set_default_stream: cuda_tnsr3d (no stream argument) follows a
    slow producer on the given non-blocking stream."""
    rng = np.random.default_rng(8)
    nel, nu, nv = 64, 4, 8
    u_host = rng.standard_normal(nel * nu ** 3)
    A, Bt, Ct = (rng.standard_normal(nu * nv) for _ in range(3))
    ref = oracle.tnsr3d(u_host, nu, nv, A, Bt, Ct, nel)
    dA, dB, dC = (torch.as_tensor(m, device="cuda") for m in (A, Bt, Ct))
    u_src = torch.as_tensor(u_host, device="cuda")
    u = torch.zeros_like(u_src)
    v = torch.zeros(nel * nv ** 3, dtype=torch.float64, device="cuda")
    q = torch.cuda.Stream()
    torch.cuda.synchronize()
    nblib.nb_set_default_stream(vp(q.cuda_stream))
    try:
        with torch.cuda.stream(q):
            torch.cuda._sleep(400_000_000)
            u.copy_(u_src)
        nblib.cuda_tnsr3d(_ptr(v), ctypes.byref(ctypes.c_int(nv)), _ptr(u),
                          ctypes.byref(ctypes.c_int(nu)), _ptr(dA), _ptr(dB), _ptr(dC),
                          ctypes.byref(ctypes.c_int(nel)))
        with torch.cuda.stream(q):
            got = v.cpu().numpy()
    finally:
        nblib.nb_set_default_stream(vp(0))
        torch.cuda.synchronize()
    assert np.abs(got - ref).max() < 1e-13 * np.abs(ref).max()


def test_vector_dropins_and_ortho(nblib):
    rng = np.random.default_rng(21)
    n = 1_000_003
    a_h, b_h, c_h = (rng.standard_normal(n) for _ in range(3))
    a, b, c = (torch.as_tensor(x, device="cuda") for x in (a_h, b_h, c_h))
    nn = ctypes.byref(ctypes.c_int(n))
    s = _stream()
    d = torch.empty_like(a)
    nblib.cuda_copy(_ptr(d), _ptr(a), nn, s)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), a_h)
    nblib.cuda_col2(_ptr(d), _ptr(b), nn, s)
    torch.cuda.synchronize()
    assert np.array_equal(d.cpu().numpy(), a_h * b_h)
    nblib.cuda_addcol3(_ptr(d), _ptr(b), _ptr(c), nn, s)
    torch.cuda.synchronize()
    _close(d.cpu().numpy(), a_h * b_h + b_h * c_h)
    nblib.cuda_rzero(_ptr(d), nn, s)
    torch.cuda.synchronize()
    assert not d.any()
    scale = np.abs(a_h).sum()
    g = nblib.cuda_glsum(_ptr(a), nn, s)
    assert abs(g - np.sum(a_h)) <= 1e-13 * scale
    g2 = nblib.cuda_glsc2(_ptr(a), _ptr(b), nn, s)
    assert abs(g2 - np.dot(a_h, b_h)) <= 1e-13 * np.abs(a_h * b_h).sum()
    # ortho: x -= glsum(x) / n, as device_ortho does with glb_n_points = n
    x = a.clone()
    shift = ctypes.c_double(-nblib.cuda_glsum(_ptr(x), nn, s) / n)
    nblib.cuda_radd(_ptr(x), ctypes.byref(shift), nn, s)
    torch.cuda.synchronize()
    ref = a_h - np.sum(a_h) / n
    assert np.abs(x.cpu().numpy() - ref).max() <= 1e-15 * np.abs(a_h).max() + 1e-15
    assert abs(nblib.cuda_glsum(_ptr(x), nn, s)) <= 1e-12 * scale


def test_fusedcg_dropins(nblib):
    rng = np.random.default_rng(5)
    n, pc = 300_007, 3
    z_h, po_h, x_h = (rng.standard_normal(n) for _ in range(3))
    P_h = [rng.standard_normal(n) for _ in range(pc)]
    al_h = rng.standard_normal(pc)
    z, po, x = (torch.as_tensor(v, device="cuda") for v in (z_h, po_h, x_h))
    p = torch.empty_like(z)
    beta = ctypes.c_double(0.37)
    nn = ctypes.byref(ctypes.c_int(n))
    nblib.cuda_fusedcg_update_p(_ptr(p), _ptr(z), _ptr(po), ctypes.byref(beta), nn)
    torch.cuda.synchronize()
    _close(p.cpu().numpy(), 0.37 * po_h + z_h)
    Pd = [torch.as_tensor(v, device="cuda") for v in P_h]
    ptrs = torch.tensor([t.data_ptr() for t in Pd], dtype=torch.int64, device="cuda")
    alpha = torch.as_tensor(al_h, device="cuda")
    nblib.cuda_fusedcg_update_x(_ptr(x), _ptr(ptrs), _ptr(alpha), ctypes.byref(ctypes.c_int(pc)),
                                nn)
    torch.cuda.synchronize()
    t = np.zeros(n)
    for j in range(pc):
        t = t + P_h[j] * al_h[j]
    _close(x.cpu().numpy(), x_h + t)
    # part2: a -= alpha c, returns sum(a b a); alpha_d(p_cur) = alpha
    a_h, b_h, c_h = (rng.standard_normal(n) for _ in range(3))
    a, b, c = (torch.as_tensor(v, device="cuda") for v in (a_h, b_h, c_h))
    al = ctypes.c_double(0.81)
    ad = torch.zeros(4, dtype=torch.float64, device="cuda")
    res = nblib.cuda_fusedcg_part2(_ptr(a), _ptr(b), _ptr(c), _ptr(ad), ctypes.byref(al),
                                   ctypes.byref(ctypes.c_int(2)), nn)
    rt = a_h - 0.81 * c_h
    _close(a.cpu().numpy(), rt)
    assert abs(res - np.sum(rt * b_h * rt)) <= 1e-13 * np.sum(np.abs(rt * b_h * rt))
    assert ad.cpu().numpy().tolist() == [0.0, 0.81, 0.0, 0.0]


def test_error_word_reported_by_its_problem(nblib):
    """A timeout recorded in one problem's error word is reported by that
    problem's next synchronising call, once; another problem's solve is
    unaffected.  The word is set from the host: no wait actually expires."""
    import neko_b200 as nb
    P1 = nb.Problem((3, 3, 3), 8)
    P2 = nb.Problem((3, 3, 3), 8)
    word = P1.field("err")
    torch.cuda.synchronize()
    assert int(word.item()) == 0
    word.fill_(1)
    torch.cuda.synchronize()
    s = _stream()
    assert nblib.nb_problem_sync(vp(P2.handle.value), s) == 0
    assert nblib.nb_problem_sync(vp(P1.handle.value), s) == 7  # NB_ERR_TIMEOUT
    assert b"expired" in nblib.nb_last_error()
    assert nblib.nb_problem_sync(vp(P1.handle.value), s) == 0  # cleared once reported
    P1.sync()
    # a solve on the problem that carries the word reports it too
    word.fill_(1)
    torch.cuda.synchronize()
    f = P2.zeros()
    f.copy_(torch.as_tensor(np.random.default_rng(1).standard_normal(P2.n), device="cuda"))
    P2.gs.op(f)
    P2.bclst.apply(f)
    mon = nb.CG(max_iter=300, abs_tol=1e-8, M=nb.Jacobi()).solve(nb.AxHelm(), P2.zeros(), f,
                                                                 P2.n, P2)
    assert mon.iter > 0
    with pytest.raises(nb.NekoB200Error) as ei:
        nb.CG(max_iter=300, abs_tol=1e-8, M=nb.Jacobi()).solve(nb.AxHelm(), P1.zeros(), f,
                                                               P1.n, P1)
    assert ei.value.status == 7
    assert int(word.item()) == 0


def test_pnpn_residual_parts(nblib):
    """The point-wise parts of the pressure and velocity residuals against
    numpy forms of src/fluid/bcknd/device/cuda/prs_res_kernel.h and
    vel_res_update_kernel.h."""
    rng = np.random.default_rng(9)
    n = 200_003
    H = {k: rng.standard_normal(n) for k in ("ta1", "ta2", "ta3", "wa1", "wa2", "wa3", "fu",
                                             "fv", "fw", "B", "p", "ur", "vr", "wr")}
    D = {k: torch.as_tensor(v, device="cuda") for k, v in H.items()}
    h1 = torch.zeros(n, dtype=torch.float64, device="cuda")
    nn = ctypes.byref(ctypes.c_int(n))
    mu, rho, dtbd = 0.013, 1.7, 3.25
    nblib.pnpn_prs_res_part1_cuda(*(_ptr(D[k]) for k in ("ta1", "ta2", "ta3", "wa1", "wa2",
                                                         "wa3", "fu", "fv", "fw", "B")),
                                  _ptr(h1), ctypes.byref(ctypes.c_double(mu)),
                                  ctypes.byref(ctypes.c_double(rho)), nn)
    torch.cuda.synchronize()
    for t, w, f in (("ta1", "wa1", "fu"), ("ta2", "wa2", "fv"), ("ta3", "wa3", "fw")):
        _close(D[t].cpu().numpy(), H[f] / rho - (H[w] * (mu / rho)) * H["B"])
    assert np.all(h1.cpu().numpy() == 1.0 / rho)
    nblib.pnpn_prs_res_part2_cuda(_ptr(D["p"]), _ptr(D["wa1"]), _ptr(D["wa2"]), _ptr(D["wa3"]),
                                  nn)
    torch.cuda.synchronize()
    p1 = -H["p"] + (H["wa1"] + H["wa2"] + H["wa3"])
    _close(D["p"].cpu().numpy(), p1)
    ta = [D[k].cpu().numpy() for k in ("ta1", "ta2", "ta3")]
    nblib.pnpn_prs_res_part3_cuda(_ptr(D["p"]), _ptr(D["ta1"]), _ptr(D["ta2"]), _ptr(D["ta3"]),
                                  ctypes.byref(ctypes.c_double(dtbd)), nn)
    torch.cuda.synchronize()
    _close(D["p"].cpu().numpy(), p1 - dtbd * (ta[0] + ta[1] + ta[2]))
    nblib.pnpn_vel_res_update_cuda(*(_ptr(D[k]) for k in ("ur", "vr", "wr")),
                                   *(_ptr(D[k]) for k in ("ta1", "ta2", "ta3")),
                                   *(_ptr(D[k]) for k in ("fu", "fv", "fw")), nn)
    torch.cuda.synchronize()
    for r, t, f in (("ur", 0, "fu"), ("vr", 1, "fv"), ("wr", 2, "fw")):
        _close(D[r].cpu().numpy(), (-H[r]) - ta[t] + H[f])
