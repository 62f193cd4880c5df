"""The C-ABI library loads and exports every entry point include/ksim_b200.h declares.

No compute is called here (no GPU on the CPU runner); calls that need a
device must fail with a status, not crash.
"""
from __future__ import annotations

import ctypes
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "ksim_b200.h"
LIB = ROOT / "ksim_b200" / "lib" / "libksim_b200.so"


def declared_functions() -> list:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(ksim_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def built_lib():
    if not LIB.exists():
        from ksim_b200.build import build
        build()
    return LIB


def test_header_declares_entry_points():
    names = declared_functions()
    for want in ("ksim_component_create", "ksim_component_sample", "ksim_component_eval_abs",
                 "ksim_program_create", "ksim_program_sample", "ksim_last_error"):
        assert want in names


def test_library_exports_every_declared_symbol(built_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(built_lib)], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_library_loads_and_reports_without_device(built_lib):
    from ksim_b200 import _abi
    L = _abi.lib()
    assert L.ksim_abi_version() == 1
    n = L.ksim_device_count()
    assert n >= 0


def test_create_without_device_is_a_status_not_a_crash(built_lib):
    from ksim_b200 import _abi, synth
    from ksim_b200.program import graph_to_dict
    L = _abi.lib()
    if L.ksim_device_count() > 0:
        pytest.skip("a device is visible")
    prog, _ = synth.htkh(1)
    descs, keep = _abi.graphs_to_descs([graph_to_dict(g) for g in prog.components[0].graphs])
    h = ctypes.c_void_p()
    st = L.ksim_component_create(descs, 2, 0, -1, ctypes.byref(h))
    assert st == _abi.KSIM_ERR_NO_DEVICE
    assert b"device" in L.ksim_last_error()
    with pytest.raises(_abi.KsimError):
        _abi.check(st)


def test_null_arguments_are_rejected(built_lib):
    from ksim_b200 import _abi
    L = _abi.lib()
    assert L.ksim_component_sample(None, None, 0, 0, 0, None) == _abi.KSIM_ERR_INVALID_ARGUMENT
    assert L.ksim_component_eval_abs(None, 0, None, 0, 0, None) == _abi.KSIM_ERR_INVALID_ARGUMENT
    assert L.ksim_program_sample(None, None, 0, 0, 0, 0, None) == _abi.KSIM_ERR_INVALID_ARGUMENT
    assert L.ksim_component_n_out(None) == -1


def test_shape_validation_before_upload():
    from ksim_b200 import _abi, synth
    from ksim_b200.program import graph_to_dict
    prog, _ = synth.htkh(2)
    graphs = [graph_to_dict(g) for g in prog.components[0].graphs]
    graphs[1]["np_params"] = np.zeros((1, 3, 1), np.uint8)   # Tnp says 2
    with pytest.raises(ValueError):
        _abi.graph_shapes_ok(graphs)
