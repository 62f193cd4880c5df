"""Generate the committed golden fixtures in tests/golden/ (run once, here).

Sources of truth, both from the reference itself:
  * the reference's numpy evaluator (``src/python/ksim/sample/evaluate.py``
    and ``exact_scalar.py``), imported from the reference tree through a stub
    ``ksim`` package (its ``__init__`` needs stim, which is absent);
  * the reference's own ``src/cpp/ksim/zx_eval.hpp``, compiled unmodified into
    ``oracle/_ref/libksim_ref.so`` (``make -C oracle``).

Per fixture program the .npz holds: the program, random parameter rows per
graph, numpy ``evaluate_flat`` amplitudes (tolerance reference), numpy
per-term numerators canonicalised (divided by 2 while all four coefficients
are even), ``zx_eval.hpp`` amplitudes (bit-exact reference), and
``zx_eval.hpp`` samples (bits and |A_k|) for two seeds in both uniform modes.

Usage: python tests/golden/make_golden.py [--ref <reference checkout>]
(default: the KSIM_REF_TREE environment variable)
"""
from __future__ import annotations

import argparse
import os
import zlib
import sys
import types
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from ksim_b200 import synth  # noqa: E402
from ksim_b200.program import save_program  # noqa: E402

OUT = Path(__file__).resolve().parent


def import_reference_numpy(ref: Path):
    src = ref / "src" / "python" / "ksim"
    pkg = types.ModuleType("ksim")
    pkg.__path__ = [str(src)]
    sys.modules["ksim"] = pkg
    sub = types.ModuleType("ksim.sample")
    sub.__path__ = [str(src / "sample")]
    sys.modules["ksim.sample"] = sub
    from ksim.sample import evaluate, exact_scalar  # type: ignore
    return evaluate, exact_scalar


def numpy_term_numerators(es, g, params):
    """Per-term (coeffs, power) exactly as evaluate_flat forms them
    (evaluate.py:32-61), before the complex cast."""
    B = params.shape[0]
    Gn = g.pf_phase_idx.shape[0]
    rs = es._gf2(g.np_params, params)
    idx = (4 * rs + g.np_phases[None]) % 8
    tv = es.ONE_PLUS_PHASES[idx]
    mask = np.arange(g.np_phases.shape[1])[None, :] < g.np_counts[:, None]
    tv = np.where(mask[None, ..., None], tv, es.IDENTITY4)
    np_c, np_p = es._prod4(tv, axis=2)
    rs = es._gf2(g.hp_params, params)
    tot = np.sum((rs * g.hp_coeffs[None]) % 8, axis=-1) % 8
    hp_c = es.UNIT_PHASES[tot]
    psi = (g.pp_psi_c[None] + es._gf2(g.pp_psi_p, params)) % 2
    phi = (g.pp_phi_c[None] + es._gf2(g.pp_phi_p, params)) % 2
    sgn = np.sum(psi * phi, axis=-1) % 2
    pp_c = (1 - 2 * sgn)[..., None] * es.IDENTITY4
    ra = es._gf2(g.ph_alpha_p, params)
    rb = es._gf2(g.ph_beta_p, params)
    al = (g.ph_alpha[None] + 4 * ra) % 8
    be = (g.ph_beta[None] + 4 * rb) % 8
    tv = es.IDENTITY4 + es.UNIT_PHASES[al] + es.UNIT_PHASES[be] - es.UNIT_PHASES[(al + be) % 8]
    mask = np.arange(g.ph_alpha.shape[1])[None, :] < g.ph_counts[:, None]
    tv = np.where(mask[None, ..., None], tv, es.IDENTITY4)
    ph_c, ph_p = es._prod4(tv, axis=2)
    static_c = es.UNIT_PHASES[g.pf_phase_idx]
    ff_c = g.pf_floatfactor.astype(np.int64)
    coeffs = es._mul4(es._mul4(es._mul4(np_c, hp_c), es._mul4(pp_c, ph_c)),
                      es._mul4(np.broadcast_to(static_c, (B, Gn, 4)),
                               np.broadcast_to(ff_c, (B, Gn, 4))))
    power = np_p + ph_p
    return coeffs, power


def canonical(coeffs, power):
    """Divide by 2 while all four coefficients are even and not all zero."""
    c = coeffs.copy()
    p = power.copy()
    for _ in range(130):
        red = np.all(c % 2 == 0, axis=-1) & np.any(c != 0, axis=-1)
        if not red.any():
            break
        c = np.where(red[..., None], c // 2, c)
        p = p + red
    return c, p


def fixture_programs():
    """(name, program, n_f) for the fixtures: random programs of several shapes
    plus the edge cases the reference path meets."""
    progs = []
    for i, (n_out, F, t) in enumerate([(3, 0, 2), (5, 0, 4), (6, 12, 6), (8, 30, 8), (4, 70, 10),
                                       (10, 20, 5)]):
        rng = np.random.default_rng(9000 + i)
        comp = synth.random_component(rng, n_out=n_out, F=F, t=t, f_prob=0.05)
        progs.append((f"rand{i}", synth.single_component_program(comp), F))
    rng = np.random.default_rng(9100)
    prog, nf = synth.multi_component_program(rng, [(2, 3, 2), (4, 6, 5), (3, 0, 3)])
    progs.append(("multi", prog, nf))
    # approximate float factors and out-of-range constant bytes
    rng = np.random.default_rng(9200)
    comp = synth.random_component(rng, n_out=4, F=6, t=5, f_prob=0.1)
    for g in comp.graphs:
        G = g.pf_phase_idx.shape[0]
        g.pf_approx = (rng.normal(size=G) + 1j * rng.normal(size=G)).astype(np.complex64)
        g.pf_has_approx = True
        g.np_phases[:] = g.np_phases + 8 * rng.integers(0, 3, size=g.np_phases.shape)
    progs.append(("approx", synth.single_component_program(comp), 6))
    # long terms (the exact / int64-wrap path)
    from ksim_b200.program import FlatComponent
    rng = np.random.default_rng(9300)
    gs = [synth.random_graph(rng, 3, 10 + k, 200, 3, 3, 30) for k in range(3)]
    comp = FlatComponent((0, 1), np.arange(10, dtype=np.int32), gs)
    progs.append(("long", synth.single_component_program(comp), 10))
    # known answers
    for k in (1, 2, 3):
        p, _ = synth.htkh(k)
        progs.append((f"htkh{k}", p, 0))
    p, _ = synth.t_depth_two()
    progs.append(("tdepth2", p, 0))
    return progs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("KSIM_REF_TREE"),
                    help="root of the reference checkout (default: $KSIM_REF_TREE)")
    a = ap.parse_args()
    if not a.ref:
        raise SystemExit("give --ref or set KSIM_REF_TREE to the reference checkout")
    ref = Path(a.ref)
    evaluate, es = import_reference_numpy(ref)
    from oracle.oracle import RefOracle, build
    build(str(ref))
    if not RefOracle.available():
        raise SystemExit("oracle/_ref not built")

    manifest = []
    for name, prog, n_f in fixture_programs():
        save_program(OUT / f"prog_{name}.npz", prog)
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        arrays = {}
        for ci, comp in enumerate(prog.components):
            F = int(np.asarray(comp.f_selection).shape[0])
            ro = RefOracle(comp.graphs, F)
            for gi, g in enumerate(comp.graphs):
                P = g.np_params.shape[2]
                pv = rng.integers(0, 2, size=(16, P)).astype(np.uint8)
                key = f"c{ci}_g{gi}"
                arrays[f"{key}_params"] = pv
                arrays[f"{key}_numpy_amp"] = evaluate.evaluate_flat(g, pv.astype(np.int64))
                if g.pf_phase_idx.shape[0]:
                    cf, pw = numpy_term_numerators(es, g, pv.astype(np.int64))
                    cf, pw = canonical(cf, pw)
                else:
                    cf = np.zeros((16, 0, 4), np.int64)
                    pw = np.zeros((16, 0), np.int64)
                arrays[f"{key}_numpy_terms"] = np.concatenate([cf, pw[..., None]], axis=-1)
                arrays[f"{key}_ref_amp"] = ro.eval(gi, pv)
            B = 512
            f = (rng.random((B, F)) < 0.1).astype(np.uint8)
            arrays[f"c{ci}_f"] = f
            for seed in (11, 2**63 + 12345):
                for mode in (0, 1):
                    bits, amp = ro.sample(f, seed, mode, return_amp=True)
                    arrays[f"c{ci}_bits_s{seed % 1000}_m{mode}"] = bits
                    arrays[f"c{ci}_amp_s{seed % 1000}_m{mode}"] = amp
        np.savez_compressed(OUT / f"golden_{name}.npz", **arrays)
        manifest.append(name)
    (OUT / "MANIFEST.txt").write_text("\n".join(manifest) + "\n")
    print("wrote", len(manifest), "fixtures")


if __name__ == "__main__":
    main()
