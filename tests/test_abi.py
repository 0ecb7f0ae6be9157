"""The C ABI library loads and exports every entry point include/*.h declares (CPU only)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
DECL = re.compile(r"^\s*(?:const\s+)?\w+\s*\*?\s*(mf_\w+)\s*\(", re.M)


def declared(header: Path):
    text = header.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(DECL.findall(text)))


def test_every_declared_symbol_is_exported(mf):
    names = []
    for h in (ROOT / "include").glob("*.h"):
        names += declared(h)
    assert len(names) >= 37
    lib = C.CDLL(str(mf.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_strings(mf):
    L = mf.lib()
    assert L.mf_version() == 2
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert L.mf_error_string(code)


def test_no_device_is_an_error_not_a_fallback(mf):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(mf.MfError) as e:
        mf.Context(0)
    assert e.value.code == -6


def test_argument_checks_without_device(mf):
    L = mf.lib()
    # scene setup rejects a degenerate lattice; the tool sampler rejects a bad spacing
    out = C.POINTER(mf.SceneStruct)()
    assert L.mf_scene_setup_ref_cut(1, 0.0, 7.0, 0.0, 0.0, 0.01, C.byref(out)) == -1
    t = mf.tool_construct((0.0, 0.01), 0.02, 0.02, 5.0, 8.0, 0.001, 0.35)
    n = C.c_int()
    assert L.mf_tool_sample(C.byref(t), 0.0, None, 0, C.byref(n)) == -1
    assert L.mf_ctx_create(0, None) == -1


def test_batch_form_entry_points_check_their_arguments(mf):
    """The batch form entry points refuse a null batch before touching a device."""
    L = mf.lib()
    k = C.c_int()
    assert L.mf_batch_set_form(None, mf.BATCH_PERSISTENT, 0, 4) == -1
    assert L.mf_batch_form(None, C.byref(k), C.byref(k)) == -1
    assert L.mf_batch_set_wait_limit(None, C.c_double(1.0)) == -1
    assert L.mf_batch_step(None, 1) == -1
    assert L.mf_batch_create(None, 1, 2, None) == -1
