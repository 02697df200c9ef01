"""Serving loop for streams of Helmholtz solve requests.

Requests (a problem shape (n, N, deformation seed), constant coefficients
h1, h2 and a right-hand side) arrive open-loop.  The server keeps every
shape's mesh, geometric factors and gather-scatter maps resident on the
device (GeometryCache, keyed by (n, lx, deformation seed)), admits requests
into a Batch while their work vectors fit the HBM budget, and advances all
admitted solves together one graph chunk at a time: a request that arrives
while others are on the GPU joins at the next chunk boundary, and a finished
request leaves at the next one (continuous batching).  Latency is measured
from arrival to the chunk boundary at which its solve was seen finished.

The one-by-one server (serve_sequential) answers the same stream with
nb_solve, one request at a time in arrival order.
"""
import collections
import math
import time

import numpy as np
import torch

from . import AxHelm, Batch, CG, FCG, Hsmg, Jacobi, NekoB200Error, Problem
from . import workloads
from ._lib import NB_ERR_OOM, NB_ERR_TIMEOUT


class GeometryCache:
    """Device-resident problems keyed by (n, lx, deformation seed)."""

    def __init__(self):
        self.problems = {}
        self.setup_s = 0.0
        self.misses = 0

    def key(self, spec):
        return (spec["n"], spec["lx"], spec["dseed"])

    def get(self, spec):
        k = self.key(spec)
        P = self.problems.get(k)
        if P is None:
            t0 = time.perf_counter()
            P = Problem((spec["n"],) * 3, spec["lx"],
                        deform=workloads.deform_amplitude(spec["dseed"]), dirichlet=True)
            self.setup_s += time.perf_counter() - t0
            self.misses += 1
            self.problems[k] = P
        return P

    def device_bytes(self):
        """Approximate HBM held by the cached problems (20 arrays of n)."""
        return sum(P.n * 8 * 20 for P in self.problems.values())

    def close(self):
        for P in self.problems.values():
            P.close()
        self.problems.clear()


class InstancePool:
    """Problem instances for the per-problem solves (hsmg slots): a slot owns
    its instance until it is released, so concurrent requests of one shape
    get distinct instances.  The first instance of a shape is the
    GeometryCache's problem; the others are created on demand and kept while
    the device has room: before a new instance is built, free extra
    instances (least recently released first) are destroyed until at least
    `reserve_gb` of device memory is free.  An instance's hsmg
    preconditioner of a precision (False for FP64, True for mixed; one of
    `variants`) is built the first time a request of that precision takes
    the instance, so an instance holds only the precisions it served."""

    def __init__(self, cache, variants=(False,), reserve_gb=16.0):
        self.cache, self.variants = cache, tuple(variants)
        self.free, self.count, self.setup_s = {}, {}, 0.0
        self.extra = []
        self.reserve = int(reserve_gb * 1e9)
        self.released = collections.OrderedDict()  # free extra instances, oldest first
        self.evicted = 0
        self.deferred = 0  # acquisitions answered "wait"
        self.built = {}  # id(instance) -> precisions whose hsmg exists

    def _make_room(self):
        while torch.cuda.mem_get_info()[0] < self.reserve and self.released:
            Pid, (k, P) = self.released.popitem(last=False)
            self.free[k].remove(P)
            self.extra.remove(P)
            self.count[k] -= 1
            self.built.pop(Pid, None)
            P.close()
            self.evicted += 1

    def _ensure(self, P, mixed):
        b = self.built.setdefault(id(P), set())
        if mixed not in b:
            t0 = time.perf_counter()
            Hsmg(mixed=mixed).init(P)
            self.setup_s += time.perf_counter() - t0
            b.add(mixed)

    def acquire(self, spec, mixed=None, wait=False):
        """An instance of spec's shape with the hsmg of precision `mixed`
        built (the first of `variants` when None).  With wait=True, None
        when every instance of the shape is in use and the device is below
        its memory reserve (the caller tries again later) rather than a new
        instance built on the room of idle ones."""
        m = self.variants[0] if mixed is None else bool(mixed)
        k = self.cache.key(spec)
        fl = self.free.setdefault(k, [])
        if fl:
            P = fl.pop()
            self.released.pop(id(P), None)
            self._ensure(P, m)
            return P
        if wait and self.count.get(k, 0) > 0 and torch.cuda.mem_get_info()[0] < self.reserve:
            self.deferred += 1
            return None
        t0 = time.perf_counter()
        if self.count.get(k, 0) == 0:
            P = self.cache.get(spec)
        else:
            self._make_room()
            P = Problem((spec["n"],) * 3, spec["lx"],
                        deform=workloads.deform_amplitude(spec["dseed"]), dirichlet=True)
            self.extra.append(P)
        self.count[k] = self.count.get(k, 0) + 1
        self.setup_s += time.perf_counter() - t0
        self._ensure(P, m)
        return P

    def release(self, spec, P):
        k = self.cache.key(spec)
        self.free.setdefault(k, []).append(P)
        if any(P is q for q in self.extra):
            self.released[id(P)] = (k, P)

    def instances(self):
        return sum(self.count.values())

    def device_bytes(self):
        """Approximate HBM of the extra instances (their hsmg levels
        included: about 30 arrays of n)."""
        return sum(P.n * 8 * 30 for P in self.extra)

    def close(self):
        for P in self.extra:
            P.close()
        self.extra.clear()


class RhsPool:
    """A few seeded right-hand sides per shape, built once (the request
    payload: a request uses variant rhs_seed % per_shape of its shape)."""

    def __init__(self, cache, per_shape=2):
        self.cache, self.per_shape, self.pool = cache, per_shape, {}

    def get(self, spec):
        P = self.cache.get(spec)
        v = spec["rhs_seed"] % self.per_shape
        k = (self.cache.key(spec), v)
        if k not in self.pool:
            f = workloads.uneven_rhs(P, 7919 * v + spec["n"])
            r0 = math.sqrt(float((f * P.field("mult") * f).sum()) / P.volume)
            self.pool[k] = (f, r0)
        return P, self.pool[k][0], self.pool[k][1]


def arrivals(rate, count, seed):
    """Open-loop Poisson arrival times (s) of `count` requests at `rate`/s."""
    gaps = np.random.default_rng(seed).exponential(1.0 / rate, count)
    return np.cumsum(gaps)


def percentiles(lat):
    a = np.sort(np.asarray(lat, dtype=np.float64))
    return {"p50_ms": float(np.percentile(a, 50) * 1e3),
            "p95_ms": float(np.percentile(a, 95) * 1e3),
            "p99_ms": float(np.percentile(a, 99) * 1e3), "max_ms": float(a[-1] * 1e3)}


# Per-request outcome of the served stream.
OK, NOT_CONVERGED, NAN, OOM_REJECTED, TIMEOUT, CANCELLED = (
    "ok", "not_converged", "nan", "oom_rejected", "timeout", "cancelled")


def serve_batched(specs, t_arr, pool, budget_bytes, rel_tol=1e-8, max_iter=5000, chunk_runs=1,
                  batch=None, stream=None, cancel=None, status=None, mode="jacobi",
                  instances=None, max_solves=64, keep_solutions=True):
    """Continuous-batching server.  Returns per-request latency (s),
    iterations, convergence flags, the span of the run (s) and the solutions
    (request index -> device tensor).

    mode "jacobi": every request is a Jacobi-PCG slot of the batched engine
    (one persistent Ax launch over all of them).  mode "fp64" / "mixed":
    requests whose spec says pc "jacobi" stay batched Jacobi slots, those
    with pc "hsmg" run as per-problem hsmg flexible-CG solves (FP64, or FP32
    smoothing with FP64 outer iteration for "mixed") on instances of
    `instances` (an InstancePool), at most `max_solves` at a time, all
    advanced together by the same run loop.

    keep_solutions=False drops each request's solution once it has been
    answered (a long stream's solutions would otherwise fill the device);
    the returned dict is then empty.

    A request may set "max_iter" in its spec.  `cancel` maps request index ->
    time (s after the start) at which the client withdraws it; a withdrawn
    request leaves the batch at the next chunk boundary.  When `status` (a
    list) is given it receives each request's outcome: ok, not_converged,
    nan, oom_rejected (its work vectors alone exceed the budget, or the
    device refused the allocation while nothing else was running), timeout
    (a bounded device wait expired; the requests then running are failed
    and the batch is rebuilt) or cancelled."""
    own = batch is None
    B = batch if batch is not None else Batch(hbm_budget=budget_bytes)
    n = len(specs)
    lat, iters, conv = [None] * n, [0] * n, [False] * n
    st = status if status is not None else [None] * n
    if len(st) < n:
        st.extend([None] * (n - len(st)))
    cancel = dict(cancel or {})
    xs, active, owned = {}, {}, {}
    waiting = collections.deque()
    nxt, done_count = 0, 0
    t0 = time.perf_counter()
    per_problem = mode in ("fp64", "mixed")

    def finish(i, outcome, now, mon=None):
        nonlocal done_count
        lat[i] = now - t_arr[i]
        st[i] = outcome
        if mon is not None:
            iters[i], conv[i] = mon.iter, mon.converged
        done_count += 1

    def release(slot):
        B.release(slot)
        i = active.pop(slot)
        if slot in owned:
            instances.release(specs[i], owned.pop(slot))
        if not keep_solutions:
            xs.pop(i, None)
        return i

    while done_count < n:
        now = time.perf_counter() - t0
        while nxt < n and t_arr[nxt] <= now:
            waiting.append(nxt)
            nxt += 1
        for i in [i for i in waiting if i in cancel and cancel[i] <= now]:
            waiting.remove(i)
            finish(i, CANCELLED, now)
        deferred = []
        while waiting:  # admission in arrival order while the budget allows
            i = waiting[0]
            sp = specs[i]
            solo = per_problem and sp.get("pc", "jacobi") == "hsmg"
            if solo and len(owned) >= max_solves:
                break
            Pi = None
            if solo:
                # when every instance of the shape is busy and the device is
                # short of memory the request waits for one to come free
                # (building one would destroy idle instances that later
                # requests need again); the requests behind it go on
                Pi = instances.acquire(sp, mixed=mode == "mixed", wait=bool(active))
                if Pi is None:
                    deferred.append(waiting.popleft())
                    continue
            P, f, r0 = pool.get(sp)
            x = torch.empty(P.n, dtype=torch.float64, device="cuda")
            try:
                if solo:
                    slot = B.submit_solve(Pi, f, x, rel_tol * r0, sp.get("max_iter", max_iter),
                                          h1=sp["h1"], h2=sp["h2"], pc="hsmg",
                                          mixed=mode == "mixed")
                else:
                    slot = B.submit(P, f, x, rel_tol * r0, sp.get("max_iter", max_iter),
                                    h1=sp["h1"], h2=sp["h2"])
            except NekoB200Error as e:
                if Pi is not None:
                    instances.release(sp, Pi)
                if e.status != NB_ERR_OOM:
                    raise
                if active:  # over budget for now: wait for slots to free
                    break
                waiting.popleft()  # cannot fit even alone
                finish(i, OOM_REJECTED, time.perf_counter() - t0)
                continue
            waiting.popleft()
            active[slot] = i
            if Pi is not None:
                owned[slot] = Pi
            xs[i] = x
        waiting.extendleft(reversed(deferred))  # deferred requests keep their places
        if not active:
            if nxt < n and not waiting:
                time.sleep(max(0.0, t_arr[nxt] - (time.perf_counter() - t0)))
            continue
        failed = None
        try:
            B.run(max_chunks=chunk_runs, stream=stream)
        except NekoB200Error as e:
            if e.status != NB_ERR_TIMEOUT:
                raise
            failed = TIMEOUT
        now = time.perf_counter() - t0
        for slot, i in list(active.items()):
            if failed is not None:
                release(slot)
                finish(i, failed, now)
                continue
            done, mon = B.result(slot)
            if i in cancel and cancel[i] <= now and not done:
                release(slot)
                finish(i, CANCELLED, now, mon)
            elif done:
                outcome = OK if mon.converged else (
                    NAN if not math.isfinite(mon.res_final) else NOT_CONVERGED)
                release(slot)
                finish(i, outcome, now, mon)
    span = time.perf_counter() - t0
    if own:
        B.close()
    return lat, iters, conv, span, xs


def serve_sequential(specs, t_arr, pool, rel_tol=1e-8, max_iter=5000, mode="jacobi"):
    """One request at a time with nb_solve, in arrival order, on the plain
    FP64 path: Jacobi-PCG (mode "jacobi", or a spec with pc "jacobi") or
    hsmg flexible CG."""
    n = len(specs)
    lat, iters, conv = [None] * n, [0] * n, [False] * n
    t0 = time.perf_counter()
    for i, sp in enumerate(specs):
        now = time.perf_counter() - t0
        if t_arr[i] > now:
            time.sleep(t_arr[i] - now)
        P, f, r0 = pool.get(sp)
        P.set_coefficients_const(sp["h1"], sp["h2"])
        x = P.zeros()
        if mode != "jacobi" and sp.get("pc", "jacobi") == "hsmg":
            solver = FCG(max_iter=max_iter, abs_tol=rel_tol * r0, M=Hsmg())
        else:
            solver = CG(max_iter=max_iter, abs_tol=rel_tol * r0, M=Jacobi())
        mon = solver.solve(AxHelm(), x, f, P.n, P)
        torch.cuda.synchronize()
        lat[i] = time.perf_counter() - t0 - t_arr[i]
        iters[i], conv[i] = mon.iter, mon.converged
    return lat, iters, conv, time.perf_counter() - t0
