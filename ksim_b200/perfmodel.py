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
