"""The jax.ffi custom calls (csrc/ffi/jr_ffi.cc, jaxrans_b200.ffi).  JAX is not installed
here, so the handlers cannot be built or run: these tests check that their absence is
reported plainly and that the handler source exports the three targets over the C ABI."""

from __future__ import annotations

import importlib.util
import re
from pathlib import Path

import pytest

from jaxrans_b200 import build as B

HAS_JAX = importlib.util.find_spec("jax") is not None


@pytest.mark.skipif(HAS_JAX, reason="JAX is installed: the handlers can be built")
def test_without_jax_nothing_is_built_and_register_says_why():
    assert B.ffi_include_dir() is None
    assert B.build_ffi() is None
    from jaxrans_b200 import ffi
    with pytest.raises(ImportError, match="install JAX"):
        ffi.register()


def test_the_handler_source_binds_the_three_targets_to_the_c_abi():
    src = B.FFI_SOURCE.read_text()
    symbols = dict(re.findall(r"XLA_FFI_DEFINE_HANDLER_SYMBOL\((\w+), (\w+),", src))
    assert symbols == {"JrResidual": "Residual", "JrJvp": "Jvp", "JrNewtonBlock": "NewtonBlock"}
    for call in ("jr_residual(", "jr_jvp(", "jr_newton_steps_async(", "jr_plan_set_stream("):
        assert call in src
    from jaxrans_b200 import ffi
    assert set(ffi._TARGETS.values()) == set(symbols)
    header = (Path(B.INCLUDE) / "jaxrans_b200.h").read_text()
    for name in re.findall(r"\b(jr_\w+)\(", src):
        assert f" {name}(" in header, name
