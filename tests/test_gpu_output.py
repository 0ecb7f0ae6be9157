"""Output path: the Usui wear evaluation on the device and the asynchronous particle dump."""
import numpy as np
import pytest

from conftest import bits_equal, rel_err
from helpers import load_oracle, load_product, perturbed_scene

pytestmark = pytest.mark.gpu

K_USUI, ALPHA_USUI = 1e-8, -2500.0


def test_usui_against_oracle(mf, orc, tmp_path):
    st = perturbed_scene(mf, ny=12, seed=41)
    ctx = load_product(mf, st)
    ctx.step(3)
    o = orc.Oracle(st["N"])
    for k in ("pos", "vel", "fc", "ft", "h", "n", "T"):
        o.set_field(k, ctx.get(k))
    t = ctx.tool_get()
    got = ctx.tool_wear_usui(K_USUI, ALPHA_USUI)
    want = o.usui(K_USUI, ALPHA_USUI, (t.vel[0], t.vel[1]))
    assert want[2] > 0.0  # particles in contact
    assert bits_equal(got[:2], want[:2])          # min and max: no rounding choices
    assert rel_err(got[2:], want[2:]) <= 1e-14    # the mean: compensated sum, other order
    # nobody in contact: zeros
    for k in ("fc", "ft"):
        ctx.set(k, np.zeros((st["N"], 2)))
    assert np.all(ctx.tool_wear_usui(K_USUI, ALPHA_USUI) == 0.0)


def test_async_dump_equals_sync_dump(mf, tmp_path):
    st = perturbed_scene(mf, ny=12, seed=42, blank_frac=0.02)
    ctx = load_product(mf, st)
    ctx.step(2)
    ctx.vtk_write(tmp_path / "sync_a.vtk")
    ctx.vtk_write_async(tmp_path / "async_a.vtk")
    # the asynchronous dump is of the state at the call, whatever runs afterwards
    ctx.step(5)
    ctx.vtk_write(tmp_path / "sync_b.vtk")
    ctx.vtk_write_async(tmp_path / "async_b.vtk")
    ctx.step(5)
    ctx.vtk_flush()
    a = (tmp_path / "sync_a.vtk").read_bytes()
    assert a == (tmp_path / "async_a.vtk").read_bytes()
    b = (tmp_path / "sync_b.vtk").read_bytes()
    assert b == (tmp_path / "async_b.vtk").read_bytes()
    assert a != b
    # blanked particles are left out
    n_live = int((ctx.get("blanked") == 0).sum())
    assert b"POINTS" in a and n_live > 0
