"""The C-ABI library: built for sm_100a, loadable, exporting every symbol the header declares."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "jaxrans_b200.h"


def declared() -> list[str]:
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void\*|double\*|const char\*)\s+(jr_\w+)\(", text, re.M)))


def test_library_builds_and_loads():
    from jaxrans_b200.build import build
    from jaxrans_b200.native import load_library
    lib = build()
    assert lib.is_file()
    load_library()


def test_every_declared_symbol_is_exported():
    from jaxrans_b200.build import build
    from jaxrans_b200.native import EXPORTS
    lib = ctypes.CDLL(str(build()))
    names = declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
    assert sorted(EXPORTS) == names


def test_errors_without_a_device_are_reported_not_crashed():
    from jaxrans_b200.native import load_library
    lib = load_library()
    assert lib.jr_plan_create(None, None) == 1          # JR_EINVAL on a null descriptor
    assert b"null" in lib.jr_last_error()


def test_batch_rejects_cases_of_different_models_on_the_host():
    """The batch check runs before any device call: an inviscid and a viscous case
    cannot share a plan (their launches differ)."""
    import ctypes as C
    from goldens import load
    from jaxrans_b200.native import PlanDesc, fill_desc, load_library
    lib = load_library()
    keep = []
    descs = (PlanDesc * 2)()
    for k, name in enumerate(["o_euler", "c_laminar"]):
        z, case, plan = load(name)
        fill_desc(descs[k], plan, case.flow, case.numerics, case.implicit, 1.0, (0.25, 0.0), keep)
    handle = C.c_void_p()
    assert lib.jr_batch_create(descs, 2, C.byref(handle)) == 1
    assert b"must share" in lib.jr_last_error()
    assert lib.jr_batch_create(descs, 0, C.byref(handle)) == 1


def test_codes_and_status_bits_match_the_header():
    """The binding's return codes and status bits are the header's."""
    from jaxrans_b200 import native
    text = HEADER.read_text()
    defines = {k: int(v) for k, v in re.findall(r"^#define (JR_\w+) (\d+)", text, re.M)}
    names = [n for n in dir(native) if n.startswith("JR_")]
    assert sorted(names) == sorted(defines)
    for name in names:
        assert getattr(native, name) == defines[name], name
    err = native.DeviceTimeout("x", native.JR_ETIMEOUT)
    assert isinstance(err, native.NativeError) and err.code == 5
