"""The drop-in claim on the GPU: our KokkosProgramSampler against the reference's caller.

``tests/golden/dropin_*.npz`` hold what the reference's own
``KokkosProgramSampler`` (src/python/ksim/sample/sampler.py:46-67, imported
unmodified) returned with its native module bound to the reference's own
zx_eval.hpp (``tests/golden/make_dropin_golden.py``): multi-component
programs with f_selection subsets and shuffled output orders, and the cfg2
stand-in.  ``ksim_b200.sampler.KokkosProgramSampler`` (the name a caller
imports after switching modules) and a hand-wired ``kokkos_sim``-style loop
over ``ksim_b200.kokkos_sim.Component`` must reproduce them bit for bit.
"""
from __future__ import annotations

import numpy as np
import pytest

from helpers import GOLDEN
from ksim_b200.program import load_program

pytestmark = pytest.mark.gpu

CASES = ["multi4", "wide2", "cfg2"]


@pytest.mark.parametrize("name", CASES)
def test_program_sampler_equals_the_reference_caller(cuda_device, name):
    from ksim_b200.sampler import KokkosProgramSampler
    prog = load_program(GOLDEN / f"dropin_prog_{name}.npz")
    d = np.load(GOLDEN / f"dropin_{name}.npz")
    got = KokkosProgramSampler(prog).sample(d["f"], int(d["seed"]))
    assert got.dtype == np.uint8 and np.array_equal(got, d["bits"])


@pytest.mark.parametrize("name", CASES)
def test_component_module_in_the_reference_loop(cuda_device, name):
    """The reference caller's steps (sampler.py:57-67) written out over our
    kokkos_sim.Component: same result."""
    from ksim_b200 import kokkos_sim
    prog = load_program(GOLDEN / f"dropin_prog_{name}.npz")
    d = np.load(GOLDEN / f"dropin_{name}.npz")
    f, seed = d["f"], int(d["seed"])
    outs = []
    for k, comp in enumerate(prog.components):
        kc = kokkos_sim.Component([g for g in comp.graphs], int(np.asarray(comp.f_selection).shape[0]))
        f_sel = np.ascontiguousarray(f[:, comp.f_selection], dtype=np.uint8)
        outs.append(np.asarray(kc.sample(f_sel, seed + 0x9E37 * k))[:, :len(comp.graphs) - 1])
    combined = np.concatenate(outs, axis=1)
    assert np.array_equal(combined[:, np.argsort(prog.output_order)], d["bits"])
