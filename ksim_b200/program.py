"""FlatProgram IR — the input format of the sampling hot path.

Field-for-field the same dataclasses as the reference's IR
(``src/python/ksim/program.py:29-53``), so a ``FlatProgram`` emitted by
``ksim.compile`` (``compile/pipeline.py:42-80``) can be handed to
:class:`ksim_b200.sampler.B200ProgramSampler` unchanged; the sampler only reads
attributes, so the reference's own dataclass instances work as well.

Per scalar graph (one per output-prefix step; G stabilizer terms, P params):

============  =========================================================
node phases   ``np_phases`` (G,Tnp) u8, ``np_params`` (G,Tnp,P) u8, ``np_counts`` (G,) i32
half-pi       ``hp_coeffs`` (G,Thp) u8 in {0,2,4,6}, ``hp_params`` (G,Thp,P)
pi products   ``pp_psi_c``/``pp_phi_c`` (G,Tpp) u8, ``pp_psi_p``/``pp_phi_p`` (G,Tpp,P)
phase pairs   ``ph_alpha``/``ph_beta`` (G,Tph) u8, their params (G,Tph,P), ``ph_counts`` (G,)
prefactor     ``pf_phase_idx`` (G,) u8, ``pf_floatfactor`` (G,4) i32, ``pf_power2`` (G,) i32,
              ``pf_approx`` (G,) c64, ``pf_has_approx`` bool
============  =========================================================

A component owns graphs ``0..n_out``: graph 0 is the normalisation, graph
``i+1`` has outputs ``0..i`` plugged and its parameter vector is
``[f (F) | m_0..m_{i-1} | trying]``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class FlatScalarGraph:
    np_phases: np.ndarray
    np_params: np.ndarray
    np_counts: np.ndarray
    hp_coeffs: np.ndarray
    hp_params: np.ndarray
    pp_psi_c: np.ndarray
    pp_psi_p: np.ndarray
    pp_phi_c: np.ndarray
    pp_phi_p: np.ndarray
    ph_alpha: np.ndarray
    ph_alpha_p: np.ndarray
    ph_beta: np.ndarray
    ph_beta_p: np.ndarray
    ph_counts: np.ndarray
    pf_phase_idx: np.ndarray
    pf_floatfactor: np.ndarray
    pf_power2: np.ndarray
    pf_approx: np.ndarray
    pf_has_approx: bool


@dataclass
class FlatComponent:
    output_indices: tuple
    f_selection: np.ndarray
    graphs: list = field(default_factory=list)


@dataclass
class FlatProgram:
    components: list
    output_order: np.ndarray
    num_outputs: int
    num_detectors: int


GRAPH_FIELDS = (
    "np_phases", "np_params", "np_counts", "hp_coeffs", "hp_params",
    "pp_psi_c", "pp_psi_p", "pp_phi_c", "pp_phi_p",
    "ph_alpha", "ph_alpha_p", "ph_beta", "ph_beta_p", "ph_counts",
    "pf_phase_idx", "pf_floatfactor", "pf_power2",
)


def graph_to_dict(g) -> dict:
    """One graph as the 19-key dict the native Component takes.

    Same keys, dtypes and contiguity as the reference's ``_graph_to_dict``
    (``sample/sampler.py:21-43``): uint8 tables, int32 counts / floatfactor /
    power2, the complex64 approx factors viewed as float32 pairs.
    """
    u8 = lambda a: np.ascontiguousarray(np.asarray(a), dtype=np.uint8)
    i32 = lambda a: np.ascontiguousarray(np.asarray(a), dtype=np.int32)
    apx = np.ascontiguousarray(np.asarray(g.pf_approx), dtype=np.complex64)
    return dict(
        np_phases=u8(g.np_phases), np_params=u8(g.np_params), np_counts=i32(g.np_counts),
        hp_coeffs=u8(g.hp_coeffs), hp_params=u8(g.hp_params),
        pp_psi_c=u8(g.pp_psi_c), pp_psi_p=u8(g.pp_psi_p),
        pp_phi_c=u8(g.pp_phi_c), pp_phi_p=u8(g.pp_phi_p),
        ph_alpha=u8(g.ph_alpha), ph_alpha_p=u8(g.ph_alpha_p),
        ph_beta=u8(g.ph_beta), ph_beta_p=u8(g.ph_beta_p), ph_counts=i32(g.ph_counts),
        pf_phase_idx=u8(g.pf_phase_idx), pf_floatfactor=i32(g.pf_floatfactor),
        pf_power2=i32(g.pf_power2), pf_approx_f32=apx.view(np.float32),
        pf_has_approx=bool(g.pf_has_approx),
    )


def save_program(path, prog: FlatProgram) -> None:
    """Write a FlatProgram to one ``.npz`` (used for fixtures and caches)."""
    arrays = {
        "output_order": np.asarray(prog.output_order, np.int32),
        "meta": np.array([len(prog.components), prog.num_outputs, prog.num_detectors], np.int64),
    }
    for ci, comp in enumerate(prog.components):
        arrays[f"c{ci}_f_selection"] = np.asarray(comp.f_selection, np.int32)
        arrays[f"c{ci}_output_indices"] = np.asarray(comp.output_indices, np.int64)
        arrays[f"c{ci}_n_graphs"] = np.array([len(comp.graphs)], np.int64)
        for gi, g in enumerate(comp.graphs):
            for name in GRAPH_FIELDS + ("pf_approx",):
                arrays[f"c{ci}_g{gi}_{name}"] = np.asarray(getattr(g, name))
            arrays[f"c{ci}_g{gi}_pf_has_approx"] = np.array([bool(g.pf_has_approx)])
    np.savez_compressed(path, **arrays)


def load_program(path) -> FlatProgram:
    z = np.load(path)
    n_comps, num_outputs, num_detectors = (int(x) for x in z["meta"])
    comps = []
    for ci in range(n_comps):
        comp = FlatComponent(tuple(int(x) for x in z[f"c{ci}_output_indices"]),
                             z[f"c{ci}_f_selection"])
        for gi in range(int(z[f"c{ci}_n_graphs"][0])):
            kw = {name: z[f"c{ci}_g{gi}_{name}"] for name in GRAPH_FIELDS + ("pf_approx",)}
            kw["pf_has_approx"] = bool(z[f"c{ci}_g{gi}_pf_has_approx"][0])
            comp.graphs.append(FlatScalarGraph(**kw))
        comps.append(comp)
    return FlatProgram(comps, z["output_order"], num_outputs, num_detectors)
