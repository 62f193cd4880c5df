"""Seeded synthetic FlatPrograms and known-answer programs.

``ksim.compile`` needs stim and pyzx_param, which this environment lacks, so
the workloads' compiled circuits cannot be produced.  This module stands in
for them with FlatPrograms whose *shapes* follow what the compiler emits
(field ranges and padding of ``compile/pipeline.py:232-397``) and whose sizes
follow a stabilizer-rank shape model:

* a component has graphs ``0..n_out``; graph ``k`` has ``P_k = F + k`` params;
* ``G_k = max(1, round(2**(0.228 t) * J))`` terms, ``J`` log-uniform in [0.5, 2]
  (the cat5 rank, ``docs/architecture.md:26`` of the reference);
* family widths ``Tnp ~ 2t + n_out/2``, ``Tph ~ t/2``, ``Thp ~ Tpp ~ n_out/4``,
  per-term counts uniform in ``[T/2, T]``; masks set each bit with
  probability ``3/P``;
* node phases mostly odd (T-gate pi/4 multiples), floatfactor coefficients in
  [-2, 2], power2 in [-4, 0] then shifted per graph so that the typical
  ``|A_k| / |A_{k-1}|`` is about 1/2 and the Bernoulli draws are not
  degenerate.

The sampled work per shot depends only on these shapes, never on the values,
so throughput measured on them is the throughput on compiled programs of the
same shape.  Known-answer programs (``htkh``, ``t_depth_two``, ``mixture``)
have exact closed-form probabilities and exercise every term family.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .program import FlatComponent, FlatProgram, FlatScalarGraph

_W = np.exp(1j * np.pi / 4)
_UNIT = np.array([_W ** k for k in range(8)])


# ---------------------------------------------------------------------------
# random graphs
# ---------------------------------------------------------------------------
def _masks(rng, G, T, P, density, active):
    """(G,T,P) uint8 masks; columns with ``active[g,t] == False`` are zero."""
    if P == 0 or T == 0:
        return np.zeros((G, T, P), np.uint8)
    m = (rng.random((G, T, P)) < density).astype(np.uint8)
    m[~active] = 0
    return m


def _counts(rng, G, T):
    if T == 0:
        return np.zeros(G, np.int32)
    lo = max(1, T // 2) if T > 0 else 0
    return rng.integers(lo, T + 1, size=G).astype(np.int32)


def random_graph(rng, G, P, Tnp, Thp, Tpp, Tph, density=None) -> FlatScalarGraph:
    """One graph with the compiler's padding rules and value ranges."""
    density = min(1.0, 3.0 / P) if (density is None and P > 0) else (density or 0.0)
    idx = np.arange

    np_counts = _counts(rng, G, Tnp)
    np_active = idx(Tnp)[None, :] < np_counts[:, None]
    # node phases: 75% odd (T-type), 20% {2,6} (S-type), 5% {0,4}
    kind = rng.random((G, Tnp))
    odd = rng.choice(np.array([1, 3, 5, 7], np.uint8), size=(G, Tnp))
    even2 = rng.choice(np.array([2, 6], np.uint8), size=(G, Tnp))
    even0 = rng.choice(np.array([0, 4], np.uint8), size=(G, Tnp))
    np_phases = np.where(kind < 0.75, odd, np.where(kind < 0.95, even2, even0)).astype(np.uint8)
    np_phases[~np_active] = 0
    np_params = _masks(rng, G, Tnp, P, density, np_active)

    hp_n = _counts(rng, G, Thp)
    hp_active = idx(Thp)[None, :] < hp_n[:, None]
    hp_coeffs = rng.choice(np.array([2, 4, 6], np.uint8), size=(G, Thp))
    hp_coeffs[~hp_active] = 0
    hp_params = _masks(rng, G, Thp, P, density, hp_active)

    pp_n = _counts(rng, G, Tpp)
    pp_active = idx(Tpp)[None, :] < pp_n[:, None]
    pp_psi_c = rng.integers(0, 2, size=(G, Tpp)).astype(np.uint8)
    pp_phi_c = rng.integers(0, 2, size=(G, Tpp)).astype(np.uint8)
    pp_psi_c[~pp_active] = 0
    pp_phi_c[~pp_active] = 0
    pp_psi_p = _masks(rng, G, Tpp, P, density, pp_active)
    pp_phi_p = _masks(rng, G, Tpp, P, density, pp_active)

    ph_counts = _counts(rng, G, Tph)
    ph_active = idx(Tph)[None, :] < ph_counts[:, None]
    ph_alpha = rng.integers(0, 8, size=(G, Tph)).astype(np.uint8)
    ph_beta = rng.integers(0, 8, size=(G, Tph)).astype(np.uint8)
    ph_alpha[~ph_active] = 0
    ph_beta[~ph_active] = 0
    ph_alpha_p = _masks(rng, G, Tph, P, density, ph_active)
    ph_beta_p = _masks(rng, G, Tph, P, density, ph_active)

    pf_phase_idx = rng.integers(0, 8, size=G).astype(np.uint8)
    ff = rng.integers(-2, 3, size=(G, 4)).astype(np.int32)
    zero = ~ff.any(axis=1)
    ff[zero, 0] = 1
    pf_power2 = rng.integers(-4, 1, size=G).astype(np.int32)
    return FlatScalarGraph(
        np_phases, np_params, np_counts, hp_coeffs, hp_params,
        pp_psi_c, pp_psi_p, pp_phi_c, pp_phi_p,
        ph_alpha, ph_alpha_p, ph_beta, ph_beta_p, ph_counts,
        pf_phase_idx, ff, pf_power2, np.ones(G, np.complex64), False)


def float_amplitude(g: FlatScalarGraph, params: np.ndarray) -> np.ndarray:
    """Approximate complex amplitude of ``g`` (float64), for calibration only.

    Evaluates the same closed form as the exact evaluator but in complex
    floating point; it is used to pick power2 shifts, never to sample."""
    params = np.asarray(params, np.int64)
    S = params.shape[0]
    G = g.pf_phase_idx.shape[0]
    if G == 0:
        return np.zeros(S, complex)

    def par(m):
        m = np.asarray(m, np.int64)
        if m.shape[-1] == 0 or m.shape[1] == 0:
            return np.zeros((S,) + m.shape[:2], np.int64)
        return np.einsum("gtp,sp->sgt", m, params[:, :m.shape[-1]]) & 1

    Tnp = g.np_phases.shape[1]
    k = (4 * par(g.np_params) + g.np_phases[None].astype(np.int64)) & 7
    f = 1 + _UNIT[k]
    f = np.where((np.arange(Tnp)[None, :] < g.np_counts[:, None])[None], f, 1)
    z = f.prod(axis=2)
    tot = ((par(g.hp_params) * g.hp_coeffs[None]) & 7).sum(axis=2) & 7
    z = z * _UNIT[tot]
    psi = (g.pp_psi_c[None] + par(g.pp_psi_p)) & 1
    phi = (g.pp_phi_c[None] + par(g.pp_phi_p)) & 1
    z = z * (1 - 2 * ((psi & phi).sum(axis=2) & 1))
    Tph = g.ph_alpha.shape[1]
    al = (g.ph_alpha[None].astype(np.int64) + 4 * par(g.ph_alpha_p)) & 7
    be = (g.ph_beta[None].astype(np.int64) + 4 * par(g.ph_beta_p)) & 7
    f = 1 + _UNIT[al] + _UNIT[be] - _UNIT[(al + be) & 7]
    f = np.where((np.arange(Tph)[None, :] < g.ph_counts[:, None])[None], f, 1)
    z = z * f.prod(axis=2)
    ff = g.pf_floatfactor.astype(float)
    ffc = ff[:, 0] + ff[:, 1] * _W + ff[:, 2] * 1j + ff[:, 3] * np.conj(_W)
    z = z * (_UNIT[g.pf_phase_idx & 7] * ffc * np.exp2(g.pf_power2.astype(float)))[None]
    if g.pf_has_approx:
        z = z * np.asarray(g.pf_approx)[None]
    return z.sum(axis=1)


def random_component(rng, n_out, F, t, f_prob=0.01, J_range=(0.5, 2.0),
                     calibrate=True, calib_samples=96) -> FlatComponent:
    """A component per the shape model (module docstring)."""
    Tnp = max(1, round(2 * t + n_out / 2))
    Tph = max(1, round(t / 2))
    Thp = max(1, round(n_out / 4))
    Tpp = max(1, round(n_out / 4))
    base = 2.0 ** (0.228 * t)
    graphs = []
    for k in range(n_out + 1):
        J = math.exp(rng.uniform(math.log(J_range[0]), math.log(J_range[1])))
        G = max(1, round(base * J))
        graphs.append(random_graph(rng, G, F + k, Tnp, Thp, Tpp, Tph))
    if calibrate and n_out > 0:
        _calibrate(rng, graphs, F, f_prob, calib_samples)
    return FlatComponent(tuple(range(n_out)), np.arange(F, dtype=np.int32), graphs)


def _calibrate(rng, graphs, F, f_prob, S):
    """Shift each graph's power2 so median |A_k| ~ median |A_0| * 2^-k."""
    f = (rng.random((S, F)) < f_prob).astype(np.int64)
    mags = []
    for k, g in enumerate(graphs):
        m = rng.integers(0, 2, size=(S, max(k - 1, 0)))
        tr = np.ones((S, 1 if k > 0 else 0), np.int64)
        params = np.hstack([f, m, tr])
        a = np.abs(float_amplitude(g, params))
        a = a[a > 0]
        mags.append(float(np.median(a)) if a.size else 1.0)
    ref = math.log2(mags[0])
    for k in range(1, len(graphs)):
        shift = round(ref - k - math.log2(mags[k]))
        graphs[k].pf_power2 = (graphs[k].pf_power2 + shift).astype(np.int32)


def single_component_program(comp: FlatComponent) -> FlatProgram:
    n_out = len(comp.graphs) - 1
    return FlatProgram([comp], np.arange(n_out, dtype=np.int32), n_out, n_out)


def multi_component_program(rng, specs, f_prob=0.01) -> tuple:
    """Several components over one shared f matrix and a shuffled output order.

    ``specs``: list of (n_out, F, t).  Returns ``(program, n_f_total)``."""
    n_f_total = sum(F for _, F, _ in specs) + 3
    comps, order = [], []
    next_out = 0
    out_ids = rng.permutation(sum(n for n, _, _ in specs))
    for n_out, F, t in specs:
        c = random_component(rng, n_out, F, t, f_prob=f_prob)
        c.f_selection = np.sort(rng.choice(n_f_total, size=F, replace=False)).astype(np.int32)
        ids = tuple(int(x) for x in out_ids[next_out:next_out + n_out])
        c.output_indices = ids
        order.extend(ids)
        next_out += n_out
        comps.append(c)
    total = len(order)
    return FlatProgram(comps, np.array(order, np.int32), total, total), n_f_total


def sample_f(rng, B, n_f, prob, chunk=1 << 16) -> np.ndarray:
    """(B, n_f) uint8 noise bits, Bernoulli(prob), generated in row chunks."""
    out = np.empty((B, n_f), np.uint8)
    for s in range(0, B, chunk):
        e = min(B, s + chunk)
        out[s:e] = rng.random((e - s, n_f), dtype=np.float32) < prob
    return out


# ---------------------------------------------------------------------------
# workload configurations
# ---------------------------------------------------------------------------
@dataclass
class Workload:
    name: str
    program: FlatProgram
    shots: int
    n_f: int
    f_prob: float
    seed: int


def _noise_prob(n_gates, F, p=1e-3):
    # X/Y/Z each with probability p after every gate; an event flips ~2 f bits
    return 0.0 if F == 0 else min(0.25, 3 * p * n_gates * 2 / (2 * F))


def config(cfg: int, index: int = 0) -> Workload:
    """Synthetic stand-in for workload ``cfg`` (1, 2, 4; 3 and 5 via helpers).

    1: 5 outputs, t=4, noiseless (F=0), 1e5 shots
    2: 40 outputs, t=12, Pauli noise p=1e-3 over 200 gates, F=64, 1e6 shots
    4: 85-qubit encoder / T layer / decoder, 16 parity outputs, t=20, F=56, 1e6 shots
    """
    seed = 1000 * cfg + index
    rng = np.random.default_rng(seed)
    if cfg == 1:
        comp = random_component(rng, n_out=5, F=0, t=4)
        return Workload("cfg1-small-5q-t4", single_component_program(comp), 100_000, 0, 0.0, seed)
    if cfg == 2:
        F = 40 + 2 * 12
        q = _noise_prob(200, F)
        comp = random_component(rng, n_out=40, F=F, t=12, f_prob=q)
        return Workload("cfg2-medium-40q-t12", single_component_program(comp), 1_000_000, F, q, seed)
    if cfg == 4:
        F = 16 + 2 * 20
        q = _noise_prob(600, F)
        comp = random_component(rng, n_out=16, F=F, t=20, f_prob=q)
        return Workload("cfg4-large-rank-85q-t20", single_component_program(comp), 1_000_000, F, q,
                        seed)
    raise ValueError(f"no single-program workload for cfg {cfg}")


def noise_model(rng, num_f: int, n_locations: int, p: float = 1e-3, flips_per_bit: int = 2):
    """A Pauli noise model of the workloads' shape: one single-qubit Pauli
    channel (X, Y, Z each with probability p) per gate location, its two
    error bits (x, z) each flipping ``flips_per_bit`` random f parameters.
    Returns (channel_probs, error_transform) in ChannelSampler's format."""
    probs = [np.array([1 - 3 * p, p, p, p], np.float64) for _ in range(n_locations)]
    T = np.zeros((num_f, 2 * n_locations), np.uint8)
    if num_f:
        for e in range(2 * n_locations):
            T[rng.choice(num_f, size=min(flips_per_bit, num_f), replace=False), e] = 1
    return probs, T


def batched_workloads(n_programs: int = 64, seed: int = 3000) -> list:
    """Workload 3: programs with qubits ~U[8,60] (all measured), t ~U[2,16],
    depth 10*qubits, p=1e-3 Pauli noise, shots log-uniform in [1e3, 1e5]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_programs):
        q = int(rng.integers(8, 61))
        t = int(rng.integers(2, 17))
        F = q + 2 * t
        prob = _noise_prob(10 * q, F)
        comp = random_component(rng, n_out=q, F=F, t=t, f_prob=prob)
        shots = int(round(math.exp(rng.uniform(math.log(1e3), math.log(1e5)))))
        out.append(Workload(f"cfg3-{i}-{q}q-t{t}", single_component_program(comp), shots, F, prob,
                            seed + 1 + i))
    return out


def serving_pool(n_programs: int = 200, seed: int = 5000) -> list:
    """Workload 5 program pool: drawn from the medium / batched / large-rank
    generators (shots are chosen per request, not here)."""
    rng = np.random.default_rng(seed)
    pool = []
    for i in range(n_programs):
        kind = int(rng.integers(0, 3))
        if kind == 0:
            n_out, t = 40, 12
        elif kind == 1:
            n_out, t = int(rng.integers(8, 61)), int(rng.integers(2, 17))
        else:
            n_out, t = 16, 20
        F = n_out + 2 * t
        prob = _noise_prob(200 if kind == 0 else (10 * n_out if kind == 1 else 600), F)
        comp = random_component(rng, n_out=n_out, F=F, t=t, f_prob=prob)
        pool.append(Workload(f"cfg5-pool-{i}", single_component_program(comp), 0, F, prob,
                             seed + 1 + i))
    return pool


# ---------------------------------------------------------------------------
# known-answer programs
# ---------------------------------------------------------------------------
def _empty_graph(G, P, Tnp=0, Thp=0, Tpp=0, Tph=0) -> FlatScalarGraph:
    z = lambda *s: np.zeros(s, np.uint8)
    return FlatScalarGraph(
        z(G, Tnp), z(G, Tnp, P), np.zeros(G, np.int32), z(G, Thp), z(G, Thp, P),
        z(G, Tpp), z(G, Tpp, P), z(G, Tpp), z(G, Tpp, P),
        z(G, Tph), z(G, Tph, P), z(G, Tph), z(G, Tph, P), np.zeros(G, np.int32),
        z(G), np.tile(np.array([1, 0, 0, 0], np.int32), (G, 1)), np.zeros(G, np.int32),
        np.ones(G, np.complex64), False)


def htkh(k: int) -> tuple:
    """H T^k H on one qubit: P(1) = sin^2(k pi/8).

    Graph 1 = (1 + w^(4m+k)) (1 + w^(4m-k)) / 4 with m the trying bit, i.e.
    (1 - cos(k pi/4) (-1)^m ... ) / 2, a two-column NodePhases product."""
    g0 = _empty_graph(1, 0)
    g1 = _empty_graph(1, 1, Tnp=2)
    g1.np_phases[0] = [k % 8, (8 - k) % 8]
    g1.np_params[0, :, 0] = 1
    g1.np_counts[0] = 2
    g1.pf_power2[0] = -2
    comp = FlatComponent((0,), np.zeros(0, np.int32), [g0, g1])
    return FlatProgram([comp], np.array([0], np.int32), 1, 1), math.sin(k * math.pi / 8) ** 2


def t_depth_two() -> tuple:
    """H T H T H on one qubit: P(1) = 1/4, as a four-term sum.

    |A(m)|^2 with A = ((1+w) + (-1)^m w(1-w)) / (2 sqrt 2) expands into four
    terms 2+sqrt2, 2-sqrt2, (-1)^m (1+i), (-1)^m (1-i), each x 2^-3; the
    (-1)^m sign is a PiProducts column (psi = m, phi = 1)."""
    g0 = _empty_graph(1, 0)
    g1 = _empty_graph(4, 1, Tpp=1)
    g1.pf_floatfactor[:] = [[2, 1, 0, 1], [2, -1, 0, -1], [1, 0, 1, 0], [1, 0, -1, 0]]
    g1.pf_power2[:] = -3
    g1.pp_psi_p[2:, 0, 0] = 1
    g1.pp_phi_c[2:, 0] = 1
    comp = FlatComponent((0,), np.zeros(0, np.int32), [g0, g1])
    return FlatProgram([comp], np.array([0], np.int32), 1, 1), 0.25


def mixture(rng, n_out: int, r: int = 2, F: int = 2, extra: bool = True) -> tuple:
    """A mixture of 2^r product distributions over n_out outputs.

    P(m | f) = 2^-r sum_g prod_j q_gj(m_j xor f_l(g,j)),
    q(b) = (2 + (-1)^b 2 cos(phi pi/4)) / 4, from two NodePhases columns with
    phases (phi, -phi).  Graph i+1 holds P(m_0..m_{i-1}, m_i = 1 | f).  With
    ``extra``, every graph also carries a HalfPi column, a PiProducts column
    and a PhasePairs column (alpha, beta in {0,4}: factor +-2) that are the same
    in every term, so they change only a global phase / sign and |A| is exact.

    Returns ``(program, n_f, prob)`` where ``prob(f_row, m_bits)`` is the exact
    joint probability of a full outcome."""
    G = 2 ** r
    phis = rng.integers(0, 8, size=(G, n_out))
    flip = rng.integers(-1, F, size=(G, n_out)) if F > 0 else -np.ones((G, n_out), int)
    graphs = []
    hp_mask = lambda P: (rng.random(P) < 0.5).astype(np.uint8)
    for k in range(n_out + 1):
        P = F + k
        Tnp = 2 * k
        g = _empty_graph(G, P, Tnp=Tnp, Thp=1 if extra else 0, Tpp=1 if extra else 0,
                         Tph=1 if extra else 0)
        for gi in range(G):
            for j in range(k):
                for c, ph in enumerate((phis[gi, j], -phis[gi, j])):
                    t = 2 * j + c
                    g.np_phases[gi, t] = ph % 8
                    g.np_params[gi, t, F + j] = 1
                    if flip[gi, j] >= 0:
                        g.np_params[gi, t, flip[gi, j]] = 1
            g.np_counts[gi] = Tnp
        g.pf_power2[:] = -r - 2 * k
        if extra and P > 0:
            hm, pm, qm, am, bm = (hp_mask(P) for _ in range(5))
            hc = int(rng.choice([2, 4, 6]))
            ac, bc = int(rng.choice([0, 4])), int(rng.choice([0, 4]))
            for gi in range(G):
                g.hp_coeffs[gi, 0] = hc
                g.hp_params[gi, 0] = hm
                g.pp_psi_p[gi, 0] = pm
                g.pp_phi_p[gi, 0] = qm
                g.pp_phi_c[gi, 0] = 1
                g.ph_alpha[gi, 0] = ac
                g.ph_beta[gi, 0] = bc
                g.ph_alpha_p[gi, 0] = am
                g.ph_beta_p[gi, 0] = bm
                g.ph_counts[gi] = 1
            g.pf_power2[:] -= 1
        elif extra:
            g.ph_alpha[:, 0] = 0
            g.ph_beta[:, 0] = 0
            g.ph_counts[:] = 1
            g.pf_power2[:] -= 1
        graphs.append(g)
    comp = FlatComponent(tuple(range(n_out)), np.arange(F, dtype=np.int32), graphs)
    prog = FlatProgram([comp], np.arange(n_out, dtype=np.int32), n_out, n_out)

    def prob(f_row, m_bits):
        tot = 0.0
        for gi in range(G):
            p = 1.0
            for j in range(n_out):
                b = int(m_bits[j]) ^ (int(f_row[flip[gi, j]]) if flip[gi, j] >= 0 else 0)
                p *= (2 + (-1) ** b * 2 * math.cos(phis[gi, j] * math.pi / 4)) / 4
            tot += p
        return tot / G

    return prog, F, prob
