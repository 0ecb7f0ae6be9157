"""The batched form: several instances advanced by one graph launch (mf_batch_*).

Each instance inside the batch runs exactly its own step sequence, so after any number of
launches its state must equal, bit for bit, that of a separate context stepped as often: with
the batched kernels (one launch per step phase for all instances; three perturbed reference
scenes, and the 64-instance parameter sweep of uneven sizes) and with the child-graph batch
that serves instances the batched kernels do not (neighbour lists).
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
    assert b.steps_per_launch == 4 and b.fused
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
    assert b.fused and b.pair_block in (64, 128, 256)
    b.close()
    # a captured graph: created and destroyed through the C ABI
    import ctypes as C
    g = C.c_void_p()
    assert mf.lib().mf_graph_capture(batched[0].h, 4, C.byref(g)) == 0 and g.value
    assert mf.lib().mf_graph_destroy(g) == 0
    assert mf.lib().mf_graph_capture(batched[0].h, 3, C.byref(g)) != 0  # odd: refused


def sweep_contexts(mf, n, precision):
    import bench

    out = []
    for p in bench.sweep_params(mf, n):
        sc = mf.Scene.from_params(p)
        c = mf.Context(0)
        c.upload_scene(sc, mf.GRID_GREEN)
        c.set_options(mf.THERMAL_BROOKSHAW, mf.JC_JOHNSON_COOK, precision)
        out.append(c)
    return out


def test_sweep_of_64_instances_equals_separate_contexts(mf):
    """The batched parameter sweep (64 instances, 3k-45k particles, speeds, rakes, depths of
    cut and JC A, B drawn per instance; mixed precision): after two launches of 4 steps with
    a tuned pair block size, every instance equals its own context bit for bit."""
    batched = sweep_contexts(mf, 64, mf.PRECISION_MIXED)
    single = sweep_contexts(mf, 64, mf.PRECISION_MIXED)
    sizes = [c.N for c in batched]
    assert min(sizes) < 8000 and max(sizes) > 30000
    b = mf.Batch(batched, steps_per_launch=0)
    assert b.fused
    steps0 = [c.status()["steps"] for c in batched]  # the tuning launches advanced the instances
    for c, s0 in zip(single, steps0):
        c.step(s0)
    b.step(2)
    for c in single:
        c.step(2 * b.steps_per_launch)
    for x, y in zip(batched, single):
        assert x.status()["steps"] == y.status()["steps"]
        assert_same(x, y)
    b.close()
    for c in batched + single:
        c.close()


def test_instances_on_neighbour_lists_take_the_child_graph_batch(mf):
    sts = scenes(mf)
    flags = mf.OPT_NEIGHBOUR_LISTS
    batched = [load_product(mf, st, precision=1, flags=flags) for st in sts]
    single = [load_product(mf, st, precision=1, flags=flags) for st in sts]
    b = mf.Batch(batched, steps_per_launch=2)
    assert not b.fused
    b.step(3)
    for c in single:
        c.step(6)
    for x, y in zip(batched, single):
        assert_same(x, y)
    b.close()


@pytest.mark.parametrize("blocks_per_sm", [0, 1, 2])
def test_persistent_batch_equals_separate_contexts(mf, blocks_per_sm):
    """The persistent form (mixed precision): K steps of every instance in one cooperative
    launch whose blocks take each phase's blocks in turn and meet at a grid barrier between
    phases. Every instance equals its own context bit for bit, over two builds of the batch's
    graph and back to the per-phase launches."""
    precision = 1
    sts = scenes(mf)
    batched = [load_product(mf, st, precision=precision) for st in sts]
    single = [load_product(mf, st, precision=precision) for st in sts]
    b = mf.Batch(batched, steps_per_launch=4)
    b.set_form(mf.BATCH_PERSISTENT, blocks_per_sm, 4)
    assert b.form == mf.BATCH_PERSISTENT and b.fused and b.steps_per_launch == 4
    assert b.blocks_per_sm >= 1 and (blocks_per_sm == 0 or b.blocks_per_sm == blocks_per_sm)
    b.step(3)
    for c in single:
        c.step(12)
    for x, y in zip(batched, single):
        assert x.status()["steps"] == 12 and x.status()["error_flags"] == 0
        assert_same(x, y)
    b.set_form(mf.BATCH_PERSISTENT, blocks_per_sm, 2)  # rebuilt: the barrier word restarts at zero
    b.step(2)
    for c in single:
        c.step(4)
    for x, y in zip(batched, single):
        assert x.status()["error_flags"] == 0
        assert_same(x, y)
    b.set_form(mf.BATCH_PHASES, 0, 2)  # and back to one launch per phase
    assert b.form == mf.BATCH_PHASES
    b.step(1)
    for c in single:
        c.step(2)
    for x, y in zip(batched, single):
        assert_same(x, y)
    b.close()


def test_persistent_sweep_of_64_instances_equals_separate_contexts(mf):
    """The 64-instance sweep (mixed precision) in the persistent form, 16 steps per launch."""
    batched = sweep_contexts(mf, 64, mf.PRECISION_MIXED)
    single = sweep_contexts(mf, 64, mf.PRECISION_MIXED)
    b = mf.Batch(batched, steps_per_launch=2)
    b.set_form(mf.BATCH_PERSISTENT, 0, 16)
    b.step(2)
    for c in single:
        c.step(32)
    for x, y in zip(batched, single):
        assert x.status()["steps"] == y.status()["steps"] == 32
        assert x.status()["error_flags"] == 0
        assert_same(x, y)
    b.close()
    for c in batched + single:
        c.close()


def test_persistent_barrier_wait_limit(mf):
    """A barrier wait that runs out ends the persistent launch early with an error the host
    reads: with a zero wait limit the first block that has to wait gives up, the barrier then
    releases no block, and every instance's status carries error bit 3; the device stays
    usable (a fresh context steps and equals a second fresh context)."""
    sts = scenes(mf)
    batched = [load_product(mf, st, precision=1) for st in sts]
    b = mf.Batch(batched, steps_per_launch=2)
    b.set_form(mf.BATCH_PERSISTENT, 0, 8)
    b.set_wait_limit(0.0)
    b.step(1)
    for x in batched:
        assert x.status()["error_flags"] & mf.ERRF_BATCH_WAIT
    b.close()
    for x in batched:
        x.close()
    fresh = [load_product(mf, sts[0], precision=1) for _ in range(2)]
    fresh[0].step(4)
    fresh[1].step(4)
    assert fresh[0].status()["error_flags"] == 0
    assert_same(fresh[0], fresh[1])
    with pytest.raises(mf.MfError):
        b2 = mf.Batch(fresh, steps_per_launch=2)
        b2.set_wait_limit(-1.0)


def test_persistent_form_refused_for_fp64_and_child_graph_batches(mf):
    sts = scenes(mf)
    fp64 = [load_product(mf, st, precision=0) for st in sts]
    b = mf.Batch(fp64, steps_per_launch=2)
    with pytest.raises(mf.MfError):
        b.set_form(mf.BATCH_PERSISTENT, 0, 4)
    b.close()
    lists = [load_product(mf, st, precision=1, flags=mf.OPT_NEIGHBOUR_LISTS) for st in sts]
    b = mf.Batch(lists, steps_per_launch=2)
    assert not b.fused
    with pytest.raises(mf.MfError):
        b.set_form(mf.BATCH_PERSISTENT, 0, 4)
    b.close()
