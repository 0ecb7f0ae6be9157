"""The batched form: several instances advanced by one graph launch (mf_batch_*).

Each instance inside the batch runs exactly its own step sequence, so after any number of
launches its state must equal, bit for bit, that of a separate context stepped as often.
"""
import numpy as np
import pytest

from conftest import bits_equal
from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "n", "idx", "blanked")


def scenes(mf):
    # uneven sizes and states: the reference scene at three resolutions, different seeds
    return [perturbed_scene(mf, ny=ny, seed=30 + ny) for ny in (8, 12, 16)]


def assert_same(a, b):
    for f in FIELDS:
        assert bits_equal(a.get(f), b.get(f)), f
    assert bits_equal(a.force_log(), b.force_log())


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_separate_contexts(mf, precision):
    sts = scenes(mf)
    batched = [load_product(mf, st, precision=precision) for st in sts]
    single = [load_product(mf, st, precision=precision) for st in sts]
    b = mf.Batch(batched, steps_per_launch=4)
    assert b.steps_per_launch == 4
    b.step(3)
    for c in single:
        c.step(12)
    for x, y in zip(batched, single):
        assert x.status()["steps"] == 12
        assert_same(x, y)
    # a host write to one instance between launches: its counts are re-primed
    v = batched[1].get("vel") * 1.01
    batched[1].set("vel", v)
    single[1].set("vel", v)
    b.step(1)
    for c in single:
        c.step(4)
    for x, y in zip(batched, single):
        assert_same(x, y)
    # a change that invalidates captured work: the batch refuses to run until rebuilt
    batched[0].set_dt(sts[0]["dt"] * 0.5)
    with pytest.raises(mf.MfError):
        b.step(1)
    b.close()


def test_batch_autotune_and_graph_capture(mf):
    sts = scenes(mf)
    batched = [load_product(mf, st) for st in sts]
    b = mf.Batch(batched, steps_per_launch=0)
    assert b.steps_per_launch in (2, 4, 8, 16)
    b.close()
    # a captured graph: created and destroyed through the C ABI
    import ctypes as C
    g = C.c_void_p()
    assert mf.lib().mf_graph_capture(batched[0].h, 4, C.byref(g)) == 0 and g.value
    assert mf.lib().mf_graph_destroy(g) == 0
    assert mf.lib().mf_graph_capture(batched[0].h, 3, C.byref(g)) != 0  # odd: refused
