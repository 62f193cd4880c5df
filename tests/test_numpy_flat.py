"""The numpy restatement of the reference's CPU sampler, pinned (CPU only).

``oracle/numpy_flat.py`` restates ``evaluate_flat`` / ``sample_flat``
(src/python/ksim/sample/evaluate.py:24-87) so the bench can time the
reference's numpy baseline where the reference tree is absent.  It must give
exactly the reference's results: the amplitudes the reference's own
``evaluate_flat`` produced for the golden fixtures (bit for bit), and the bits
its ``sample_flat`` drew for fixed f rows and seeds (``numpy_sample.npz``,
made by ``tests/golden/make_numpy_golden.py``).
"""
from __future__ import annotations

import warnings

import numpy as np
import pytest

from helpers import GOLDEN, golden_names, load_golden, same_bits
from ksim_b200 import synth


@pytest.mark.parametrize("name", golden_names())
def test_amplitudes_equal_the_reference_numpy(name):
    from oracle import numpy_flat as nf
    prog, d = load_golden(name)
    for ci, comp in enumerate(prog.components):
        for gi, g in enumerate(comp.graphs):
            got = nf.evaluate_flat(g, d[f"c{ci}_g{gi}_params"])
            assert same_bits(got, d[f"c{ci}_g{gi}_numpy_amp"]), (name, ci, gi)


def _fixture_programs():
    progs = {name: load_golden(name)[0] for name in golden_names()}
    for cfg in (1, 2):
        progs[f"cfg{cfg}"] = synth.config(cfg).program
    return progs


def test_sample_flat_equals_the_reference_draws():
    from oracle import numpy_flat as nf
    d = np.load(GOLDEN / "numpy_sample.npz")
    progs = _fixture_programs()
    names = [str(n) for n in d["names"]]
    assert set(names) == set(progs)
    for name in names:
        with warnings.catch_warnings():
            warnings.simplefilter("ignore", RuntimeWarning)  # the reference divides by |A| = 0 too
            got = nf.sample_flat(progs[name], d[f"{name}_f"], np.random.default_rng(int(d[f"{name}_seed"])))
        assert np.array_equal(got, d[f"{name}_bits"]), name


def test_omega_table_and_product():
    from oracle import numpy_flat as nf
    w = np.exp(1j * np.pi / 4)
    basis = np.array([1, w, 1j, np.conj(w)])
    for k in range(8):
        assert abs(nf.W_POW[k] @ basis - w ** k) < 1e-12
    rng = np.random.default_rng(1)
    x, y = rng.integers(-50, 50, (2, 100, 4))
    assert np.allclose(nf.zmul(x, y) @ basis, (x @ basis) * (y @ basis))
