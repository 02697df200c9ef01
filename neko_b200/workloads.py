"""Seeded synthetic workloads of the benchmarks (inputs only).

* unit box 8^3, lx = 8, zero Dirichlet on every face,
  f = 3 pi^2 sin(pi x) sin(pi y) sin(pi z) + xi, xi ~ N(0, 1e-3) per local
  point made continuous by gs_add(xi) * mult; b = gs_add(B f), masked
  (the shape of examples/poisson/driver.f90 + setup.f90).
* periodic box [0, 2 pi]^3, 32^3 elements, lx = 8, GLL points
  displaced by 0.05 sin of the other two coordinates; f = sum over integer
  wave vectors 0 < |k| <= 4 (half space) of a_k cos(k.x) + b_k sin(k.x)
  with a_k, b_k ~ N(0, 1); b_local = B f, de-meaned as ortho does
  (src/math/operators.f90:349-368), then gs_add.
"""
import math

import numpy as np
import torch

UNIT_BOX_8 = dict(nel=(8, 8, 8), lx=8, lo=(0.0,) * 3, hi=(1.0,) * 3, periodic=(False,) * 3,
                  deform=0.0, dirichlet=True, rel_tol=1e-10, max_iter=500)
PERIODIC_BOX_32 = dict(nel=(32, 32, 32), lx=8, lo=(0.0,) * 3, hi=(2 * math.pi,) * 3,
                       periodic=(True,) * 3, deform=0.05, dirichlet=False, rel_tol=1e-8,
                       max_iter=5000)


def fourier_modes(kmax=4):
    ks = []
    for a in range(-kmax, kmax + 1):
        for b in range(-kmax, kmax + 1):
            for c in range(-kmax, kmax + 1):
                if a * a + b * b + c * c == 0 or a * a + b * b + c * c > kmax * kmax:
                    continue
                first = next(v for v in (a, b, c) if v != 0)
                if first > 0:
                    ks.append((a, b, c))
    return np.array(ks, dtype=np.float64)


def fourier_field(x, y, z, seed, kmax=4):
    """sum_k a_k cos(k.x) + b_k sin(k.x) on arrays (numpy or torch; numpy
    inputs are evaluated with torch on the host threads and returned as
    numpy)."""
    ks = fourier_modes(kmax)
    amp = np.random.default_rng(seed).standard_normal((len(ks), 2))
    is_np = not isinstance(x, torch.Tensor)
    if is_np:
        x, y, z = (torch.from_numpy(np.ascontiguousarray(v)) for v in (x, y, z))
    f = torch.zeros_like(x)
    for (k1, k2, k3), (a, b) in zip(ks, amp):
        ph = k1 * x + k2 * y + k3 * z
        f += a * torch.cos(ph) + b * torch.sin(ph)
    return f.numpy() if is_np else f


def periodic_box_rhs(x, y, z, B, seed):
    """B f de-meaned over local points (before gs)."""
    bl = B * fourier_field(x, y, z, seed)
    return bl - bl.sum() / bl.numel() if isinstance(bl, torch.Tensor) else bl - bl.sum() / bl.size


def unit_box_pointwise(x, y, z, xi_cont):
    pi = math.pi
    if isinstance(x, torch.Tensor):
        s = torch.sin
    else:
        s = np.sin
    return 3 * pi ** 2 * s(pi * x) * s(pi * y) * s(pi * z) + xi_cont


# --- batched and served streams: uneven Helmholtz problems -----------------------------------
N_DEFORM_SEEDS = 8


def deform_amplitude(dseed):
    """Deformation amplitude of deformation seed `dseed` (U[0, 0.1])."""
    return float(np.random.default_rng(1000 + dseed).uniform(0.0, 0.1))


def uneven_specs(count=512, seed=4):
    """Problem descriptions of the batched / served workloads: a box of n^3
    elements with n ~ U{2..16}, N ~ {5, 7, 9} (lx = N + 1), h1 ~ U[0.5, 2],
    h2 ~ U[0, 100], a deformation seed (8 seeds, amplitude U[0, 0.1] each),
    zero Dirichlet on the box faces and a Fourier-mode right-hand side.
    The preconditioner per problem ("pc"): Jacobi for the boxes of at most
    3^3 elements, where the multigrid's fixed cost per iteration outweighs
    its savings, hsmg for the others."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        out.append(dict(n=int(rng.integers(2, 17)), lx=int(rng.choice([5, 7, 9])) + 1,
                        h1=float(rng.uniform(0.5, 2.0)), h2=float(rng.uniform(0.0, 100.0)),
                        dseed=int(rng.integers(0, N_DEFORM_SEEDS)), rhs_seed=int(seed * 100003 + i)))
        out[-1]["pc"] = "jacobi" if out[-1]["n"] <= 3 else "hsmg"
    return out


def uneven_rhs(P, rhs_seed, kmax=3):
    """B f with f a seeded Fourier series on the unit box (device tensor),
    assembled and masked."""
    x, y, z, B = (P.field(k) for k in ("x", "y", "z", "B"))
    two_pi = 2 * math.pi
    f = B * fourier_field(two_pi * x, two_pi * y, two_pi * z, rhs_seed, kmax)
    f = f.contiguous()
    P.gs.op(f)
    P.bclst.apply(f)
    return f


# --- unstructured hexahedral meshes -------------------------------------------
def cube_rotations():
    """The 24 proper rotations of the reference cube as (axis permutation,
    flips): local corner c' of the rotated element is corner
    (c'[perm[d]] ^ flips[d])_d of the original."""
    import itertools
    out = []
    for perm in itertools.permutations(range(3)):
        inv = sum(1 for a in range(3) for b in range(a + 1, 3) if perm[a] > perm[b])
        for flips in itertools.product((0, 1), repeat=3):
            if (inv + sum(flips)) % 2 == 0:
                out.append((perm, flips))
    return out


def box_mesh(nel, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0), periodic=(False, False, False),
             rotate_seed=None):
    """An nel[0] x nel[1] x nel[2] box as an unstructured mesh: vertex ids
    (nelv, 8) and coordinates (nelv, 8, 3) in symmetric vertex order, x
    fastest; in periodic directions the last grid plane takes the ids of the
    first.  With rotate_seed each element's local frame is turned by a
    random proper rotation of the cube (same hexahedron, rotated numbering),
    so neighbouring elements meet with arbitrary relative orientation."""
    nx, ny, nz = nel
    G = [n + (0 if p else 1) for n, p in zip(nel, periodic)]
    h = [(hi[d] - lo[d]) / nel[d] for d in range(3)]
    rots = cube_rotations()
    rng = np.random.default_rng(rotate_seed) if rotate_seed is not None else None
    ids, xyz = [], []
    for ez in range(nz):
        for ey in range(ny):
            for ex in range(nx):
                base = (ex, ey, ez)
                vid, vx = [], []
                for v in range(8):
                    c = (v & 1, (v >> 1) & 1, v >> 2)
                    g = [base[d] + c[d] for d in range(3)]
                    w = [g[d] % G[d] if periodic[d] else g[d] for d in range(3)]
                    vid.append(1 + w[0] + G[0] * (w[1] + G[1] * w[2]))
                    vx.append([lo[d] + h[d] * g[d] for d in range(3)])
                if rng is not None:
                    perm, flips = rots[rng.integers(len(rots))]
                    order = []
                    for v in range(8):
                        c = (v & 1, (v >> 1) & 1, v >> 2)
                        o = [c[perm[d]] ^ flips[d] for d in range(3)]
                        order.append(o[0] + 2 * o[1] + 4 * o[2])
                    vid = [vid[q] for q in order]
                    vx = [vx[q] for q in order]
                ids.append(vid)
                xyz.append(vx)
    return np.array(ids, dtype=np.int32), np.array(xyz, dtype=np.float64)


def hub_mesh(nel, k, rotate_seed=None):
    """box_mesh(nel) plus k elements that share only the first vertex of
    element 0 with the rest of the mesh (each a copy of element 0's
    hexahedron with seven new vertex ids): one point with more copies than
    a warp has lanes, as at the singular vertices of unstructured meshes."""
    ids, xyz = box_mesh(nel, rotate_seed=rotate_seed)
    nid = int(ids.max()) + 1
    extra = [[int(ids[0, 0])] + list(range(nid + 7 * e, nid + 7 * e + 7)) for e in range(k)]
    return (np.concatenate([ids, np.array(extra, dtype=np.int32)]),
            np.concatenate([xyz, np.repeat(xyz[:1], k, axis=0)]))
