"""Checkpoint / resume (mf_state_save / mf_state_load) and device-memory field access."""
import numpy as np
import pytest

from conftest import bits_equal
from helpers import load_product, perturbed_scene

pytestmark = pytest.mark.gpu

FIELDS = ("pos", "vel", "S", "rho", "T", "eps_pl", "eps_pl_dot", "fc", "ft", "n", "pos_t", "vel_t", "rho_t", "S_t",
          "T_t", "blanked", "hash", "id")


def snapshot(ctx):
    return {f: ctx.get(f) for f in FIELDS}


@pytest.mark.parametrize("grid_kind", [0, 1])
def test_resume_continues_bit_for_bit(mf, tmp_path, grid_kind):
    st = perturbed_scene(mf, ny=12, seed=51, blank_frac=0.01)
    a = load_product(mf, st, grid_kind=grid_kind)
    a.step(5)
    a.state_save(tmp_path / "s.bin")
    a.step(5)
    b = load_product(mf, st, grid_kind=grid_kind)
    b.state_load(tmp_path / "s.bin")
    assert b.status()["steps"] == 5
    b.step(5)
    sa, sb = snapshot(a), snapshot(b)
    for f in FIELDS:
        assert bits_equal(sa[f], sb[f]), f


def test_mixed_resume(mf, tmp_path):
    """The mixed form (sorted every step) resumes bit for bit; on neighbour lists a loaded
    state starts with a sort (the lists are not saved), so the resumed run follows the
    uninterrupted one to FP32 summation order."""
    from conftest import rel_err
    st = perturbed_scene(mf, ny=12, seed=52, blank_frac=0.01)
    for flags, exact in ((0, True), (mf.OPT_NEIGHBOUR_LISTS, False)):
        a = load_product(mf, st, precision=mf.PRECISION_MIXED, flags=flags)
        a.step(5)
        a.state_save(tmp_path / "m.bin")
        a.step(5)
        b = load_product(mf, st, precision=mf.PRECISION_MIXED, flags=flags)
        b.state_load(tmp_path / "m.bin")
        b.step(5)
        oa, ob = np.argsort(a.get("id")), np.argsort(b.get("id"))
        for f in ("pos", "vel", "S", "rho", "T", "eps_pl", "blanked"):
            x, y = a.get(f)[oa], b.get(f)[ob]
            if exact:
                assert bits_equal(x, y), (f, flags)
            else:
                assert rel_err(x, y) < 1e-5, (f, rel_err(x, y))


def test_corrupted_or_foreign_files_are_refused(mf, tmp_path):
    st = perturbed_scene(mf, ny=12, seed=52)
    a = load_product(mf, st)
    a.step(2)
    path = tmp_path / "s.bin"
    a.state_save(path)
    raw = bytearray(path.read_bytes())
    b = load_product(mf, st)
    before = snapshot(b)
    cases = {"flipped": raw[:len(raw) // 2] + bytes([raw[len(raw) // 2] ^ 0x40]) + raw[len(raw) // 2 + 1:],
             "truncated": raw[:-100], "empty": b""}
    for name, data in cases.items():
        bad = tmp_path / f"{name}.bin"
        bad.write_bytes(bytes(data))
        with pytest.raises(mf.MfError) as e:
            b.state_load(bad)
        assert e.value.code == mf.MF_ERR_CORRUPT, name
    # a state of another particle count
    other = load_product(mf, perturbed_scene(mf, ny=8, seed=53))
    with pytest.raises(mf.MfError) as e:
        other.state_load(path)
    assert e.value.code == mf.MF_ERR_CORRUPT
    after = snapshot(b)
    for f in FIELDS:  # nothing was applied
        assert bits_equal(before[f], after[f]), f


def test_fields_to_and_from_device_memory(mf):
    torch = pytest.importorskip("torch")
    st = perturbed_scene(mf, ny=12, seed=54, blank_frac=0.05)
    ctx = load_product(mf, st)
    ctx.step(2)
    n = st["N"]
    dev = torch.device("cuda", 0)
    pos = torch.empty((n, 2), dtype=torch.float64, device=dev)
    ctx.get_device("pos", pos.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(pos.cpu().numpy(), ctx.get("pos"))
    blk = torch.empty(n, dtype=torch.float64, device=dev)
    ctx.get_device("blanked", blk.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(blk.cpu().numpy(), ctx.get("blanked"))
    # writes through the caller's stream
    s = torch.cuda.Stream(device=dev)
    vel = torch.full((n, 2), 1e-5, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    ctx.set_device("vel", vel.data_ptr(), s.cuda_stream)
    assert np.all(ctx.get("vel") == 1e-5)
    fixed = torch.zeros(n, dtype=torch.float64, device=dev)
    fixed[:10] = 1.0
    torch.cuda.synchronize()
    ctx.set_device("fixed", fixed.data_ptr())
    assert np.array_equal(ctx.get("fixed"), fixed.cpu().numpy())
    bad = torch.full((n,), 0.5, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    with pytest.raises(mf.MfError):
        ctx.set_device("fixed", bad.data_ptr())
