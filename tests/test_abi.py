"""The C-ABI library: loads without a GPU, exports every entry point of
include/collatz.h, and runs its host-only parts."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "collatz.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(collatz_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import collatz_b200 as cb
    L = cb.lib()
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n


def test_status_strings():
    import collatz_b200 as cb
    assert cb.status_string(0) == "ok"
    assert "argument" in cb.status_string(cb.E_ARG)


def test_create_without_device_fails_loudly():
    import collatz_b200 as cb
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(cb.CollatzError) as e:
        cb.Verifier(26)
    assert e.value.status == cb.E_NODEV


def test_bad_config_rejected():
    import collatz_b200 as cb
    cfg = cb.Config()
    cb.lib().collatz_config_default(ctypes.byref(cfg))
    assert (cfg.maxbits, cfg.range_k) == (45, 24)
    cfg.maxbits = 200
    h = ctypes.c_void_p()
    assert cb.lib().collatz_create(ctypes.byref(cfg), ctypes.byref(h)) == cb.E_ARG


def test_step1_pairs_rejects_bad_tuple():
    import collatz_b200 as cb
    with pytest.raises(cb.CollatzError):
        cb.step1_pairs(26, 3, 17, 12, 9, 1, 0)


def test_step1_pairs_layout():
    import collatz_b200 as cb
    leaves = cb.step1_pairs(26, 3, 2, 2, 9, 1, 0)
    assert len(leaves) == 1370
    mbi = 16
    for bi, base, number in leaves:
        assert base < (1 << mbi) and base % 2 == 1
        assert 0 <= bi < 16


def test_int_peak_rejects_null_arguments():
    """collatz_int_peak validates its arguments before touching a device."""
    import collatz_b200 as cb
    out = cb.IntPeakC()
    assert cb.lib().collatz_int_peak(None, 1, ctypes.byref(out)) == cb.E_ARG
    assert cb.lib().collatz_int_peak(None, 1, None) == cb.E_ARG
