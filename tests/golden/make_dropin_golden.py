"""Generate tests/golden/dropin_*.npz: the reference's own caller, run here (once).

The reference's ``src/python/ksim/sample/sampler.py`` (``KokkosProgramSampler``:
per-component Component construction, the f_selection gather, the per-component
seed ``seed + 0x9E37 k``, the concatenation and the argsort(output_order)
permutation, sampler.py:46-67) is imported unmodified from the reference tree
through a stub ``ksim`` package, with its native module ``kokkos_sim`` bound to
the reference's own ``zx_eval.hpp`` compiled into ``oracle/_ref`` (the
kokkos_sim loop restated in ``oracle/ref_driver.cpp``).  The programs are
built with the reference's own ``FlatProgram`` dataclasses.  Each fixture keeps
the program, the f rows, the seed and the reference caller's output, so the
GPU drop-in (``ksim_b200.sampler.KokkosProgramSampler``) is compared with the
reference's caller on a machine without the reference tree.

Usage: python tests/golden/make_dropin_golden.py [--ref <reference checkout>]
(default: the KSIM_REF_TREE environment variable)
"""
from __future__ import annotations

import argparse
import os
import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ksim_b200 import synth  # noqa: E402
from ksim_b200.program import save_program  # noqa: E402

OUT = Path(__file__).resolve().parent


def import_reference_sampler(ref: Path):
    """The reference's ksim.program and ksim.sample.sampler modules, with
    kokkos_sim bound to oracle/_ref."""
    from oracle import oracle as orc
    orc.build(str(ref))
    if not orc.RefOracle.available():
        raise SystemExit("oracle/_ref not built")

    class Component:  # kokkos_sim.Component over the reference's zx_eval.hpp
        def __init__(self, graphs, num_f):
            self._o = orc.RefOracle(graphs, num_f)
            self.n_out = len(graphs) - 1

        def sample(self, f_sel, seed):
            return self._o.sample(f_sel, int(seed), 0)

    shim = types.ModuleType("kokkos_sim")
    shim.Component = Component
    sys.modules["kokkos_sim"] = shim
    src = ref / "src" / "python" / "ksim"
    pkg = types.ModuleType("ksim")
    pkg.__path__ = [str(src)]
    sys.modules["ksim"] = pkg
    sub = types.ModuleType("ksim.sample")
    sub.__path__ = [str(src / "sample")]
    sys.modules["ksim.sample"] = sub
    import ksim.program as kprog  # type: ignore
    from ksim.sample import sampler as ksampler  # type: ignore
    return kprog, ksampler


def as_reference_program(kprog, prog):
    """The same program in the reference's own dataclasses."""
    comps = []
    for c in prog.components:
        graphs = [kprog.FlatScalarGraph(**{k: getattr(g, k) for k in g.__dataclass_fields__}) for g in c.graphs]
        comps.append(kprog.FlatComponent(output_indices=tuple(c.output_indices),
                                         f_selection=np.asarray(c.f_selection), graphs=graphs))
    return kprog.FlatProgram(components=comps, output_order=np.asarray(prog.output_order),
                             num_outputs=prog.num_outputs, num_detectors=prog.num_detectors)


def cases():
    """(name, program, n_f columns, shots)."""
    out = []
    rng = np.random.default_rng(7100)
    prog, nf = synth.multi_component_program(rng, [(4, 10, 4), (6, 20, 6), (3, 0, 3), (9, 40, 9)])
    out.append(("multi4", prog, nf, 3000))
    rng = np.random.default_rng(7200)
    prog, nf = synth.multi_component_program(rng, [(12, 70, 8), (2, 5, 2)])
    out.append(("wide2", prog, nf, 2000))
    w = synth.config(2)
    out.append(("cfg2", w.program, w.n_f, 2000))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("KSIM_REF_TREE"),
                    help="root of the reference checkout (default: $KSIM_REF_TREE)")
    a = ap.parse_args()
    if not a.ref:
        raise SystemExit("give --ref or set KSIM_REF_TREE to the reference checkout")
    kprog, ksampler = import_reference_sampler(Path(a.ref))
    rng = np.random.default_rng(20261205)
    for name, prog, n_f, B in cases():
        f = synth.sample_f(rng, B, n_f, 0.05)
        seed = int(rng.integers(0, 2**62))
        ref_prog = as_reference_program(kprog, prog)
        bits = np.asarray(ksampler.KokkosProgramSampler(ref_prog).sample(f, seed), np.uint8)
        save_program(OUT / f"dropin_prog_{name}.npz", prog)
        np.savez_compressed(OUT / f"dropin_{name}.npz", f=f, seed=np.array(seed, np.int64), bits=bits)
        print(f"dropin_{name}: {bits.shape}")


if __name__ == "__main__":
    main()
