"""Host logic of the served stream's instance pool, without a GPU: the
problem instances and the device's free memory are stand-ins.  A shape's
first instance is the geometry cache's problem and is never destroyed; extra
instances are reused when free and, when a new one must be built while the
device is short of memory, free extra instances are destroyed oldest-first
until the reserve is met."""
import pytest

from neko_b200 import serve


class FakeProblem:
    made = 0

    def __init__(self, nel, lx, deform=0.0, dirichlet=True):
        FakeProblem.made += 1
        self.n = nel[0] ** 3 * lx ** 3
        self.closed = False

    def close(self):
        self.closed = True


class FakeHsmg:
    built = []

    def __init__(self, mixed=False):
        self.mixed = mixed

    def init(self, P):
        FakeHsmg.built.append((id(P), self.mixed))


class FakeCache:
    def __init__(self):
        self.problems = {}

    def key(self, spec):
        return (spec["n"], spec["lx"], spec["dseed"])

    def get(self, spec):
        return self.problems.setdefault(self.key(spec), FakeProblem((spec["n"],) * 3, spec["lx"]))


@pytest.fixture
def pool(monkeypatch):
    free = {"bytes": 100 * 10 ** 9}
    monkeypatch.setattr(serve, "Problem", FakeProblem)
    monkeypatch.setattr(serve, "Hsmg", FakeHsmg)
    monkeypatch.setattr(serve.torch.cuda, "mem_get_info", lambda: (free["bytes"], 180 * 10 ** 9))
    return serve.InstancePool(FakeCache(), variants=(False, True), reserve_gb=16.0), free


def spec(n, lx=5, dseed=0):
    return {"n": n, "lx": lx, "dseed": dseed}


def test_first_instance_is_cached_problem_and_reused(pool):
    p, _ = pool
    a = p.acquire(spec(3))
    assert a is p.cache.get(spec(3))
    p.release(spec(3), a)
    assert p.acquire(spec(3)) is a
    assert p.instances() == 1


def test_concurrent_requests_get_distinct_instances(pool):
    p, _ = pool
    a, b, c = (p.acquire(spec(4)) for _ in range(3))
    assert len({id(a), id(b), id(c)}) == 3
    assert p.instances() == 3


def test_eviction_when_short_of_memory(pool):
    p, free = pool
    s1, s2 = spec(3), spec(6)
    a = p.acquire(s1)
    extra = [p.acquire(s1) for _ in range(3)]  # three extra instances of s1
    for q in extra:
        p.release(s1, q)
    p.release(s1, a)
    free["bytes"] = 10 * 10 ** 9  # below the 16 GB reserve
    first = p.acquire(s2)       # the cache's problem of s2: no eviction needed
    assert p.evicted == 0
    q = p.acquire(s2)           # an extra instance: free extras are destroyed first
    assert q is not first
    assert p.evicted == 3 and all(x.closed for x in extra)
    assert not a.closed        # the cache's problem is kept
    assert p.instances() == 1 + 2


def test_in_use_instances_are_never_evicted(pool):
    p, free = pool
    s = spec(5)
    held = [p.acquire(s) for _ in range(3)]
    free["bytes"] = 1
    p.acquire(spec(7))
    p.acquire(spec(7))
    assert p.evicted == 0 and not any(h.closed for h in held)


def test_precisions_built_on_first_use(pool):
    p, _ = pool
    FakeHsmg.built.clear()
    a = p.acquire(spec(3), mixed=True)
    assert FakeHsmg.built == [(id(a), True)]
    p.release(spec(3), a)
    assert p.acquire(spec(3), mixed=True) is a
    assert len(FakeHsmg.built) == 1  # nothing rebuilt
    p.release(spec(3), a)
    p.acquire(spec(3), mixed=False)
    assert FakeHsmg.built[-1] == (id(a), False) and len(FakeHsmg.built) == 2


def test_wait_instead_of_building_when_short(pool):
    p, free = pool
    s = spec(5)
    a = p.acquire(s)                 # the cache's problem
    b = p.acquire(s)                 # an extra one while memory allows
    free["bytes"] = 1
    assert p.acquire(s, wait=True) is None and p.deferred == 1
    p.release(s, b)
    assert p.acquire(s, wait=True) is b   # a free instance is always handed out
    assert p.acquire(spec(9), wait=True) is not None  # a shape's first instance is built
    assert not a.closed
