"""Algorithmic work of one shot: the roofline numerator.

The sampling kernels are bound by 32-bit integer ALU work.  Per shot the
work is fixed by the program's structure alone (never by the sampled values):
for every graph k and term g it walks the term's columns.  The int32 operation
counts below are the irreducible work of the formulation in
``ksim_b200/csrc/zring.cuh`` with W 64-bit parameter words:

=================  ===========================================================
NodePhases column  parity 3W (AND, XOR-fold, popcount) + sign 2
                   + conditional-negate-add of 4 int64 (16) [+ halving 8 + 1
                   on the columns the valuation schedule marks]
HalfPi column      parity 3W + select-add 2
PiProducts column  two parities 6W + 4
PhasePairs column  two parities 6W + three rotated int64x4 adds (48)
                   + valuation / halving 12
per term           phase rotations, sign, floatfactor product (16 int64
                   multiplies ~ 48 + 24 adds), renormalisation, header: 160
per graph          parameter-vector masks and sums: 4W + 8
=================  ===========================================================

HBM bytes per shot: the f row (``F`` bytes) in and the output row out.
"""
from __future__ import annotations

import numpy as np


def _np_reduce_flags(phases: np.ndarray) -> int:
    nu, red = 0, 0
    for ph in phases:
        j = int(ph) & 3
        if j == 0:
            continue
        nu += 1 if j & 1 else 2
        if nu >= 4:
            nu -= 4
            red += 1
    return red


def graph_work(g, W: int) -> dict:
    """Column counts and int32 ops of one graph for one shot."""
    G = int(g.pf_phase_idx.shape[0])
    P = int(g.np_params.shape[2]) if g.np_params.ndim == 3 else 1
    n_np = n_hp = n_pp = n_ph = n_red = 0
    for t in range(G):
        cnp = max(0, int(g.np_counts[t]))
        cph = max(0, int(g.ph_counts[t]))
        n_np += cnp
        n_ph += cph
        n_red += _np_reduce_flags(g.np_phases[t, :cnp] & 7)
        if g.hp_coeffs.shape[1]:
            live = (g.hp_coeffs[t] & 7) != 0
            if P:
                live &= g.hp_params[t].any(axis=1)
            else:
                live &= False
            n_hp += int(live.sum())
        if g.pp_psi_c.shape[1]:
            psi0 = ((g.pp_psi_c[t] & 1) == 0) & ~(g.pp_psi_p[t].any(axis=1) if P else False)
            phi0 = ((g.pp_phi_c[t] & 1) == 0) & ~(g.pp_phi_p[t].any(axis=1) if P else False)
            n_pp += int((~(psi0 | phi0)).sum())
    ops = (n_np * (3 * W + 18) + n_red * 9 + n_hp * (3 * W + 2) + n_pp * (6 * W + 4)
           + n_ph * (6 * W + 60) + G * 160 + 4 * W + 8)
    return {"terms": G, "np": n_np, "hp": n_hp, "pp": n_pp, "ph": n_ph, "ops": ops}


def words_for(comp) -> int:
    supported = (1, 2, 3, 4, 5, 6, 8, 10, 12, 16)
    F = int(np.asarray(comp.f_selection).shape[0])
    bits = max([F + len(comp.graphs) - 1] + [int(g.np_params.shape[2]) for g in comp.graphs] + [1])
    need = (bits + 1 + 63) // 64  # plus the constant-one bit
    return next(w for w in supported if w >= need)


def program_work(prog) -> dict:
    """Per-shot totals over all components and graphs of a FlatProgram."""
    tot = {"terms": 0, "np": 0, "hp": 0, "pp": 0, "ph": 0, "ops": 0, "graphs": 0,
           "in_bytes": 0, "out_bytes": 0}
    for comp in prog.components:
        W = words_for(comp)
        for g in comp.graphs:
            w = graph_work(g, W)
            for k in ("terms", "np", "hp", "pp", "ph", "ops"):
                tot[k] += w[k]
            tot["graphs"] += 1
        tot["in_bytes"] += int(np.asarray(comp.f_selection).shape[0])
    tot["out_bytes"] = int(len(prog.output_order))
    tot["columns"] = tot["np"] + tot["hp"] + tot["pp"] + tot["ph"]
    return tot
