"""Algorithmic work of one shot: the roofline numerator.

The sampling kernels are bound by 32-bit integer ALU / multiply-add issue.
Per shot the work is fixed by the program's structure alone (never by the
sampled values): every graph k is evaluated once and every term of it once.
The int32 operation counts come from the packer (``ksim_work_model`` in
``include/ksim_b200.h``, costs listed in ``ksim_b200/csrc/image.cpp``), which
knows each term's path: 32-bit words for terms whose values are proven
below 2^31, 32-bit NodePhases and 64-bit words for the rest when only the
NodePhases block is, 64-bit words otherwise, the reference's step-by-step
arithmetic (84 int32 operations per Z[w] product) on the exact path.

HBM bytes per shot: the f row (``F`` bytes) in and the output row out.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from .program import graph_to_dict


def component_work(comp) -> dict:
    """int32 ops per shot and terms per path of one FlatComponent."""
    graphs = [graph_to_dict(g) for g in comp.graphs]
    descs, keep = _abi.graphs_to_descs(graphs)
    ops = ctypes.c_double()
    paths = (ctypes.c_int64 * 4)()
    F = int(np.asarray(comp.f_selection).shape[0])
    _abi.check(_abi.lib().ksim_work_model(descs, len(graphs), F, ctypes.byref(ops), paths))
    del keep
    return {"ops": float(ops.value), "narrow_terms": paths[0], "wide_terms": paths[1],
            "exact_terms": paths[2], "hybrid_terms": paths[3]}


def reference_op_model(prog) -> float:
    """int32 operations per shot of the reference's own algorithm
    (zx_eval.hpp:75-181 run once per graph, kokkos_sim.cpp:214-230): per
    term g of graph k, cnt_np[g] + cnt_ph[g] + 3 Z[w] products (NodePhases and
    PhasePairs columns, HalfPi, prefactor phase, floatfactor) at 84 int32 ops
    each (16 int64 multiplies at 3, 12 int64 adds at 2, the reduce at 12), and
    (Tnp + Thp + 2 Tpp + 2 Tph) * ceil(P_k / 64) 64-bit parity words at 5 ops
    each (AND, POPC and accumulate on 64-bit words).  It describes the
    reference's step-by-step work, not the reformulated work the kernels run
    (``component_work``), which is several times smaller."""
    total = 0.0
    for comp in prog.components:
        for g in comp.graphs:
            G = int(g.pf_phase_idx.shape[0])
            if G == 0:
                continue
            Tnp = int(g.np_phases.shape[1]) if g.np_phases.ndim > 1 else 0
            Thp = int(g.hp_coeffs.shape[1]) if g.hp_coeffs.ndim > 1 else 0
            Tpp = int(g.pp_psi_c.shape[1]) if g.pp_psi_c.ndim > 1 else 0
            Tph = int(g.ph_alpha.shape[1]) if g.ph_alpha.ndim > 1 else 0
            P = int(g.np_params.shape[2]) if g.np_params.ndim > 2 else 0
            words = max(1, -(-P // 64))
            zmul = float(np.sum(np.asarray(g.np_counts, np.int64)) +
                         np.sum(np.asarray(g.ph_counts, np.int64)) + 3 * G)
            parw = float(G * (Tnp + Thp + 2 * Tpp + 2 * Tph) * words)
            total += 84.0 * zmul + 5.0 * parw
    return total


def program_work(prog) -> dict:
    """Per-shot totals over all components and graphs of a FlatProgram."""
    tot = {"terms": 0, "ops": 0.0, "graphs": 0, "in_bytes": 0, "out_bytes": 0,
           "narrow_terms": 0, "wide_terms": 0, "exact_terms": 0, "hybrid_terms": 0}
    for comp in prog.components:
        w = component_work(comp)
        for k in ("ops", "narrow_terms", "wide_terms", "exact_terms", "hybrid_terms"):
            tot[k] += w[k]
        tot["terms"] += sum(int(g.pf_phase_idx.shape[0]) for g in comp.graphs)
        tot["graphs"] += len(comp.graphs)
        tot["in_bytes"] += int(np.asarray(comp.f_selection).shape[0])
    tot["out_bytes"] = int(len(prog.output_order))
    return tot
