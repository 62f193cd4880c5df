"""Generate tests/golden/numpy_sample.npz from the reference's sample_flat (run once, here).

The reference's numpy sampler (src/python/ksim/sample/evaluate.py:69-87) is
imported from the reference tree through a stub ``ksim`` package (its
``__init__`` needs stim, which is absent) and run on the committed fixture
programs and on the cfg1 / cfg2 stand-ins with seeded f rows and a seeded
``numpy.random.default_rng``.  The fixture keeps the f rows, the seed and the
reference's bits, so the numpy restatement under oracle/ is pinned to the
reference wherever the reference tree is absent.

Usage: python tests/golden/make_numpy_golden.py [--ref <reference checkout>]
(default: the KSIM_REF_TREE environment variable)
"""
from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

from golden.make_golden import import_reference_numpy  # noqa: E402
from helpers import golden_names, load_golden  # noqa: E402
from ksim_b200 import synth  # noqa: E402

OUT = Path(__file__).resolve().parent / "numpy_sample.npz"


def cases():
    """(name, program, n_f columns, shots, f probability)."""
    out = []
    for name in golden_names():
        prog, d = load_golden(name)
        n_f = max([int(np.max(c.f_selection)) + 1 for c in prog.components if len(c.f_selection)] or [0])
        out.append((name, prog, n_f, 300, 0.05))
    for cfg in (1, 2):
        w = synth.config(cfg)
        out.append((f"cfg{cfg}", w.program, w.n_f, 120, w.f_prob))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("KSIM_REF_TREE"),
                    help="root of the reference checkout (default: $KSIM_REF_TREE)")
    a = ap.parse_args()
    if not a.ref:
        raise SystemExit("give --ref or set KSIM_REF_TREE to the reference checkout")
    evaluate, _ = import_reference_numpy(Path(a.ref))
    rng = np.random.default_rng(20261204)
    arrays = {}
    names = []
    for name, prog, n_f, B, p in cases():
        f = synth.sample_f(rng, B, n_f, p)
        seed = int(rng.integers(0, 2**31))
        bits = np.asarray(evaluate.sample_flat(prog, f, np.random.default_rng(seed)), np.uint8)
        arrays[f"{name}_f"] = f
        arrays[f"{name}_seed"] = np.array(seed, np.int64)
        arrays[f"{name}_bits"] = bits
        names.append(name)
    arrays["names"] = np.array(names)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({len(names)} cases)")


if __name__ == "__main__":
    main()
