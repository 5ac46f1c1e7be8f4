"""Batched instances (cc_batch_create) on the GPU: the batch equals the same
union built by the caller, and on a first step from rest (same query radius
everywhere, no refresh) every instance equals its own independent solver bit
for bit: colouring, detection and sweeps do not mix instances."""
import numpy as np
import pytest

from clothcraft_b200 import native, scenes
from clothcraft_b200.vbd import VbdSolver

pytestmark = pytest.mark.gpu

LANES = 8


def instances():
    return scenes.config2_instances(seed=11, count=4, sides=(12, 24), pitch=1.0)


def settings(sc):
    s = sc.settings
    s.refresh_fraction = 1.0  # refresh only if every vertex clips: same decision for batch and instances
    return s.to_c()


def lanes(solver):
    assert native.load().cc_solver_set_lanes(solver.h, LANES) == 0
    return solver


def test_batch_equals_caller_built_union():
    inst = instances()
    b = lanes(VbdSolver.batch(inst))
    u = lanes(VbdSolver(scenes.batch_scene(inst)))
    assert b.n == u.n and b.total == u.total
    assert b.instances() == [(sum(s.n for s in inst[:k]), inst[k].n) for k in range(len(inst))]
    st = inst[0].settings.to_c()
    x = np.concatenate([s.x0 for s in inst])
    v = np.zeros_like(x)
    xb, vb, tb = x.copy(), v.copy(), 0.0
    xu, vu, tu = x.copy(), v.copy(), 0.0
    for _ in range(3):
        xb, vb, tb, mb = b.step(xb, vb, tb, st)
        xu, vu, tu, mu = u.step(xu, vu, tu, st)
        assert np.array_equal(xb, xu) and np.array_equal(vb, vu)
        assert mb["contact_terms"] == mu["contact_terms"]


def test_first_step_of_each_instance_equals_its_own_solver():
    inst = instances()
    st = settings(inst[0])
    b = lanes(VbdSolver.batch(inst))
    x = np.concatenate([s.x0 for s in inst])
    xb, _, _, mb = b.step(x, np.zeros_like(x), 0.0, st)
    for (first, count), sc in zip(b.instances(), inst):
        g = lanes(VbdSolver(sc))
        xi, _, _, mi = g.step(sc.x0, sc.v0, 0.0, st)
        assert np.array_equal(xb[first:first + count], xi)
    assert mb["colors"] == max(1, mb["colors"])
