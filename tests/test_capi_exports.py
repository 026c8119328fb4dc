"""The C-ABI library loads and exports every entry point declared in include/tmsolve.h
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

from tmsolve import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "tmsolve.h")).read()
    return sorted(set(re.findall(r"^\s*(?:tm_status|void|int32_t|int64_t)\s+(tm_\w+)\s*\(", src, re.M)))


def test_header_lists_entry_points():
    names = declared()
    assert "tm_solve" in names and "tm_anand_screen" in names and "tm_create" in names
    assert set(_lib.EXPORTED) <= set(names)


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    missing = [n for n in declared() if not hasattr(L, n)]
    assert not missing, missing


def test_no_device_is_an_error_not_a_fallback():
    """Without a GPU the library refuses with TM_NO_DEVICE (there is no CPU path)."""
    import torch
    if torch.cuda.is_available():
        return
    from tmsolve.packages import fcbga_c1
    from tmsolve.solver import DeviceModel
    try:
        DeviceModel(fcbga_c1())
    except _lib.TmError as e:
        assert e.status == _lib.TM_NO_DEVICE
    else:
        raise AssertionError("tm_create succeeded without a device")


def declared_arity():
    """Parameter count of every entry point in include/tmsolve.h (`(void)` counts as none)."""
    src = open(os.path.join(ROOT, "include", "tmsolve.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for m in re.finditer(r"^\s*(?:tm_status|void|int32_t|int64_t|const char\s*\*)\s*(tm_\w+)\s*\(([^;]*?)\)\s*;", src, re.M | re.S):
        params = m.group(2).strip()
        out[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return out


def test_binding_argument_counts_match_header():
    """Every ctypes argtypes list the binding sets has exactly as many entries as the C declaration."""
    L = _lib.load()
    ar = declared_arity()
    bad = {}
    for n in _lib.EXPORTED:
        at = getattr(L, n).argtypes
        if at is not None and n in ar and len(at) != ar[n]:
            bad[n] = (len(at), ar[n])
    assert not bad, bad
