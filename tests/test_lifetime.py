"""CPU checks of the Python binding's ownership rule: a system's LNV solvers are destroyed before
the system, whichever Python object is closed (or finalised) first.  A fake library records the
C calls; no GPU and no CUDA call is involved."""
import ctypes

import numpy as np
import pytest

import cq_b200


class FakeLib:
    def __init__(self):
        self.calls = []
        self.next = 0x1000
        self.live_solvers = set()

    def _handle(self, out_ref):
        self.next += 0x10
        out_ref._obj.value = self.next
        return self.next

    def cq_system_create(self, *args):
        h = self._handle(args[-1])
        self.calls.append(("system_create", h))
        return 0

    def cq_system_destroy(self, h):
        # the C library refuses while solvers of the system are alive
        if self.live_solvers:
            self.calls.append(("system_destroy_refused", h.value))
            return cq_b200.CQ_ERR_STATE
        self.calls.append(("system_destroy", h.value))
        return 0

    def cq_lnv_params_default(self, p):
        return 0

    def cq_lnv_create(self, sys_h, ids, ne, params, out_ref):
        h = self._handle(out_ref)
        self.live_solvers.add(h)
        self.calls.append(("lnv_create", h))
        return 0

    def cq_lnv_destroy(self, h):
        assert h.value in self.live_solvers, "solver destroyed twice"
        self.live_solvers.discard(h.value)
        self.calls.append(("lnv_destroy", h.value))
        return 0

    def cq_last_error(self):
        return b"fake"


@pytest.fixture
def fake(monkeypatch):
    f = FakeLib()
    f.objects = []
    monkeypatch.setattr(cq_b200, "_lib", f)
    yield f
    # fake handles must never reach the real library, even if a failed test keeps objects alive
    for o in f.objects:
        o._h = ctypes.c_void_p()


def _make(fake):
    coords = np.zeros((2, 3)); cell = np.ones(3) * 10.0
    g = cq_b200.System(coords, cell, [4, 4], [10.0] * 11)
    ids = {n: i for i, n in enumerate(cq_b200.LNV_RANGE_NAMES)}
    objs = (g, cq_b200.LNV(g, ids, 1.0), cq_b200.LNV(g, ids, 1.0))
    fake.objects.extend(objs)
    return objs


@pytest.mark.parametrize("system_first", [True, False])
def test_solvers_are_destroyed_before_their_system(fake, system_first):
    g, a, b = _make(fake)
    if system_first:
        g.close(); a.close(); b.close()
    else:
        a.close(); g.close(); b.close()
    names = [c[0] for c in fake.calls]
    assert names.count("lnv_destroy") == 2 and names.count("system_destroy") == 1
    assert "system_destroy_refused" not in names
    assert names.index("system_destroy") > max(i for i, n in enumerate(names) if n == "lnv_destroy")
    assert not fake.live_solvers


def test_finaliser_order_does_not_matter(fake):
    g, a, b = _make(fake)
    g.__del__()                      # as the cycle collector may do: the system first
    a.__del__(); b.__del__()
    assert not fake.live_solvers
    assert [c[0] for c in fake.calls].count("system_destroy") == 1
