"""numpy restatement of the reference's CPU sampler (test infrastructure only).

The reference ships a pure-numpy evaluator and sampler over the FlatProgram IR,
``evaluate_flat`` / ``sample_flat`` (src/python/ksim/sample/evaluate.py:24-87)
on the exact Z[w] helpers of src/python/ksim/sample/exact_scalar.py:19-66.
That code cannot travel with this repository (it lives in the reference
tree), so this module restates the same algorithm, step for step where the
result depends on it:

* GF(2) parities as an int64 contraction of the 0/1 masks with the parameter
  rows, reduced mod 2 (exact_scalar.py:64-66);
* NodePhases: factors 1 + w^((4 par + phase) mod 8), columns past
  ``np_counts`` replaced by 1, multiplied in column order with one
  "halve if all four even and not all zero" step after every product,
  the padded columns included (exact_scalar.py:44-55, evaluate.py:32-37);
* HalfPi: w^(sum (par * coeff mod 8) mod 8) (evaluate.py:39-41);
* PiProducts: the sign (-1)^(sum psi phi) (evaluate.py:43-46);
* PhasePairs: factors 1 + w^a + w^b - w^(a+b) with the same product and
  halving schedule as NodePhases (evaluate.py:48-53);
* the unreduced product of the four families with w^idx and the floatfactor,
  the complex cast a + b w + c i + d conj(w) times 2^power, the prefactor
  2^power2 (or the approximate factor) and numpy's own sum over terms
  (evaluate.py:55-66, exact_scalar.py:58-61);
* ``sample_flat``: per component, graph 0's |A| then one ``rng.random(B)``
  draw per output, bit = u < p1 / prev, prev = bit ? p1 : prev - p1, outputs
  permuted by argsort(output_order) (evaluate.py:69-87).

Integer work is exact mod 2^64 whatever the order of the products; the
floating-point steps use the same numpy operations in the same order, so
amplitudes and bits equal the reference's.  Pinned by
``tests/test_numpy_flat.py`` against fixtures made from the reference's own
module.  Only tests/ and bench.py's CPU baseline use it.
"""
from __future__ import annotations

import numpy as np

_OMEGA = np.exp(1j * np.pi / 4)


def _powers_of_omega() -> np.ndarray:
    """(8, 4) int64: w^k in the basis (1, w, i, conj w) for k = 0..7."""
    out = np.zeros((8, 4), np.int64)
    z = np.array([1, 0, 0, 0], np.int64)
    for k in range(8):
        out[k] = z
        a, b, c, d = z
        z = np.array([d, a, b, -c], np.int64)  # multiply by w
    return out


W_POW = _powers_of_omega()
ONE_PLUS = W_POW.copy()
ONE_PLUS[:, 0] += 1
ONE = np.array([1, 0, 0, 0], np.int64)


def zmul(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Z[w] product on the last axis (basis 1, w, i, conj w), wrapping int64."""
    xa, xb, xc, xd = x[..., 0], x[..., 1], x[..., 2], x[..., 3]
    ya, yb, yc, yd = y[..., 0], y[..., 1], y[..., 2], y[..., 3]
    return np.stack([xa * ya + xb * yd - xc * yc + xd * yb,
                     xa * yb + xb * ya + xc * yd + xd * yc,
                     xa * yc + xb * yb + xc * ya - xd * yd,
                     xa * yd - xb * yc - xc * yb + xd * ya], axis=-1)


def halve_once(z: np.ndarray, power: np.ndarray) -> tuple:
    """One renormalisation step where all four are even and not all zero."""
    even = np.all(z % 2 == 0, axis=-1) & np.any(z != 0, axis=-1)
    return np.where(even[..., None], z // 2, z), power + even.astype(power.dtype)


def column_product(factors: np.ndarray) -> tuple:
    """Product over axis -2 of (..., T, 4) factors, halving after each product."""
    T = factors.shape[-2]
    lead = factors.shape[:-2]
    if T == 0:
        return np.broadcast_to(ONE, lead + (4,)).copy(), np.zeros(lead, np.int64)
    z = factors[..., 0, :].astype(np.int64)
    power = np.zeros(lead, np.int64)
    for t in range(1, T):
        z = zmul(z, factors[..., t, :].astype(np.int64))
        z, power = halve_once(z, power)
    return z, power


def parities(masks: np.ndarray, rows: np.ndarray) -> np.ndarray:
    """(G, T, P) masks and (B, P) parameter rows -> (B, G, T) parities."""
    return np.einsum("gtp,bp->bgt", masks.astype(np.int64), rows.astype(np.int64)) % 2


def _live(counts: np.ndarray, T: int) -> np.ndarray:
    return (np.arange(T)[None, :] < np.asarray(counts)[:, None])[None, ..., None]


def evaluate_flat(g, rows: np.ndarray) -> np.ndarray:
    """Complex amplitude (B,) of one FlatScalarGraph for parameter rows (B, P)."""
    B = rows.shape[0]
    G = g.pf_phase_idx.shape[0]
    if G == 0:
        return np.zeros(B, np.complex128)
    # NodePhases
    par = parities(g.np_params, rows)
    f = ONE_PLUS[(4 * par + g.np_phases[None]) % 8]
    f = np.where(_live(g.np_counts, g.np_phases.shape[1]), f, ONE)
    z_np, pw_np = column_product(f)
    # HalfPi
    par = parities(g.hp_params, rows)
    z_hp = W_POW[np.sum((par * g.hp_coeffs[None]) % 8, axis=-1) % 8]
    # PiProducts
    psi = (g.pp_psi_c[None] + parities(g.pp_psi_p, rows)) % 2
    phi = (g.pp_phi_c[None] + parities(g.pp_phi_p, rows)) % 2
    z_pp = (1 - 2 * (np.sum(psi * phi, axis=-1) % 2))[..., None] * ONE
    # PhasePairs
    al = (g.ph_alpha[None] + 4 * parities(g.ph_alpha_p, rows)) % 8
    be = (g.ph_beta[None] + 4 * parities(g.ph_beta_p, rows)) % 8
    f = ONE + W_POW[al] + W_POW[be] - W_POW[(al + be) % 8]
    f = np.where(_live(g.ph_counts, g.ph_alpha.shape[1]), f, ONE)
    z_ph, pw_ph = column_product(f)
    # prefactor and complex cast
    pre = zmul(np.broadcast_to(W_POW[g.pf_phase_idx], (B, G, 4)),
               np.broadcast_to(g.pf_floatfactor.astype(np.int64), (B, G, 4)))
    z = zmul(zmul(zmul(z_np, z_hp), zmul(z_pp, z_ph)), pre)
    power = pw_np + pw_ph
    amp = (z[..., 0] + z[..., 1] * _OMEGA + z[..., 2] * 1j + z[..., 3] * np.conj(_OMEGA))
    amp = amp * np.exp2(power.astype(np.float64))
    if g.pf_has_approx:
        return np.sum(amp * g.pf_approx[None] * np.exp2(g.pf_power2)[None], axis=-1)
    return np.sum(amp * np.exp2(g.pf_power2.astype(np.float64))[None], axis=-1)


def sample_flat(prog, f_params: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """(B, num_outputs) sampled bits of a FlatProgram (one draw per output)."""
    B = f_params.shape[0]
    cols = []
    for comp in prog.components:
        n_out = len(comp.graphs) - 1
        f = f_params[:, comp.f_selection].astype(np.int64)
        m = np.zeros((B, n_out), np.int64)
        prev = np.abs(evaluate_flat(comp.graphs[0], f))
        for i, g in enumerate(comp.graphs[1:]):
            rows = np.hstack([f, m[:, :i], np.ones((B, 1), np.int64)])
            p1 = np.abs(evaluate_flat(g, rows))
            bit = rng.random(B) < (p1 / prev)
            m[:, i] = bit
            prev = np.where(bit, p1, prev - p1)
        cols.append(m)
    out = np.concatenate(cols, axis=1) if cols else np.zeros((B, 0), np.int64)
    return out[:, np.argsort(prog.output_order)]
