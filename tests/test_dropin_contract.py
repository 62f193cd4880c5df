"""The reference's own caller against this package's kokkos_sim module (CPU).

Runs only where the reference checkout is available (KSIM_REF_TREE).  The
reference's ``sample/sampler.py`` is imported unmodified with
``sys.modules["kokkos_sim"] = ksim_b200.kokkos_sim`` (the one-line switch a
maintainer makes to run the reference's caller on this package).  On a machine without a GPU the native Component cannot upload, so
this checks the contract up to the device: the reference constructs
``Component(graphs, num_f)`` with the dicts of its ``_graph_to_dict``
(sampler.py:21-43), those dicts are byte-identical to this package's
``graph_to_dict`` and pack through the C ABI's host-side packer
(``ksim_work_model``), and the failure to reach a device surfaces as this
package's error, not as a signature or type mismatch.  The numerical side of
the same claim runs on the GPU (``tests/test_gpu_dropin.py``).
"""
from __future__ import annotations

import os
import sys
import types
from pathlib import Path

import numpy as np
import pytest

from helpers import GOLDEN
from ksim_b200.program import graph_to_dict, load_program

REF = os.environ.get("KSIM_REF_TREE")
pytestmark = pytest.mark.skipif(not REF or not Path(REF).exists(),
                                reason="KSIM_REF_TREE does not name a reference checkout")


@pytest.fixture()
def reference_sampler(monkeypatch):
    from ksim_b200 import kokkos_sim
    src = Path(REF) / "src" / "python" / "ksim"
    pkg = types.ModuleType("ksim")
    pkg.__path__ = [str(src)]
    sub = types.ModuleType("ksim.sample")
    sub.__path__ = [str(src / "sample")]
    for name in [n for n in sys.modules if n == "ksim" or n.startswith("ksim.")]:
        monkeypatch.delitem(sys.modules, name)
    monkeypatch.setitem(sys.modules, "ksim", pkg)
    monkeypatch.setitem(sys.modules, "ksim.sample", sub)
    monkeypatch.setitem(sys.modules, "kokkos_sim", kokkos_sim)
    import importlib
    return importlib.import_module("ksim.sample.sampler")


def test_reference_dicts_are_ours_and_pack(reference_sampler):
    from ksim_b200 import _abi, perfmodel  # noqa: F401
    prog = load_program(GOLDEN / "dropin_prog_multi4.npz")
    for comp in prog.components:
        for g in comp.graphs:
            theirs = reference_sampler._graph_to_dict(g)
            ours = graph_to_dict(g)
            assert set(theirs) == set(ours)
            for k in theirs:
                a, b = np.asarray(theirs[k]), np.asarray(ours[k])
                assert a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a, b), k
        # the C ABI's host packer accepts the reference's dicts as they are
        work = perfmodel.component_work(comp)
        assert work["ops"] > 0


def test_reference_caller_reaches_our_component(reference_sampler):
    from ksim_b200 import _abi
    prog = load_program(GOLDEN / "dropin_prog_multi4.npz")
    if _abi.lib().ksim_device_count() > 0:
        pytest.skip("a GPU is visible: tests/test_gpu_dropin.py covers the numbers")
    with pytest.raises(_abi.KsimError) as e:
        reference_sampler.KokkosProgramSampler(prog)
    assert e.value.status == _abi.KSIM_ERR_NO_DEVICE
