"""Generate tests/golden/noise_*.npz from the reference's ChannelSampler (run once, here).

The reference's ``src/python/ksim/compile/channels.py`` imports only numpy,
so it is loaded straight from the reference tree.  For each noise model (the
reference's own channel constructors, a seeded random GF(2) error_transform)
the fixture holds the channel probabilities and transform as passed to
``ChannelSampler``, seeded random parity sets over f, the exact probability of
each parity computed from the reference's precomputed sparse channel data
(``_precompute_sparse``, after its channel simplification), and the parity
frequencies of 200,000 shots drawn by the reference's ``sample``.

Usage: python tests/golden/make_noise_golden.py [--ref <reference checkout>]
(default: the KSIM_REF_TREE environment variable)
"""
from __future__ import annotations

import argparse
import os
import importlib.util
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def load_channels(ref: Path):
    path = ref / "src" / "python" / "ksim" / "compile" / "channels.py"
    spec = importlib.util.spec_from_file_location("ref_channels", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ref_channels"] = mod  # dataclasses look their module up
    spec.loader.exec_module(mod)
    return mod


def models(ch, rng):
    out = {}
    # 1: independent bit flips, one error bit per f column plus shared ones
    probs = [ch.error_probs(p) for p in rng.uniform(1e-3, 0.2, 12)]
    T = (rng.random((9, 12)) < 0.25).astype(np.uint8)
    out["flips"] = (probs, T)
    # 2: single-qubit Pauli channels (2 error bits each)
    probs = [ch.pauli_channel_1_probs(*rng.uniform(1e-3, 0.05, 3)) for _ in range(20)]
    T = (rng.random((14, 40)) < 0.15).astype(np.uint8)
    out["pauli1"] = (probs, T)
    # 3: two-qubit Pauli channels (4 error bits) and heralded channels (3 bits)
    probs = [ch.pauli_channel_2_probs(*rng.uniform(1e-4, 4e-3, 15)) for _ in range(6)]
    probs += [ch.heralded_pauli_channel_1_probs(*rng.uniform(1e-3, 0.05, 4)) for _ in range(4)]
    n_e = 6 * 4 + 4 * 3
    T = (rng.random((70, n_e)) < 0.08).astype(np.uint8)
    out["pauli2_heralded"] = (probs, T)
    return out


def exact_from_sparse(sparse, cols):
    prod = 1.0
    for p_fire, cond_cdf, xor_pats in sparse:
        p_out = p_fire * np.diff(np.concatenate([[0.0], cond_cdf]))
        odd = (xor_pats[:, cols].sum(axis=1) % 2) == 1
        prod *= 1.0 - 2.0 * float(p_out[odd].sum())
    return (1.0 - prod) / 2.0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("KSIM_REF_TREE"),
                    help="root of the reference checkout (default: $KSIM_REF_TREE)")
    a = ap.parse_args()
    if not a.ref:
        raise SystemExit("give --ref or set KSIM_REF_TREE to the reference checkout")
    ch = load_channels(Path(a.ref))
    rng = np.random.default_rng(20261203)
    for name, (probs, T) in models(ch, rng).items():
        num_f = T.shape[0]
        sets = [[j] for j in range(num_f)]
        sets += [sorted(rng.choice(num_f, size=int(rng.integers(2, 5)), replace=False).tolist())
                 for _ in range(12)]
        sampler = ch.ChannelSampler(probs, T, seed=7)
        exact = [exact_from_sparse(sampler._sparse_data, s) for s in sets]
        draws = sampler.sample(200_000)
        freq = [float((draws[:, s].sum(axis=1) % 2).mean()) for s in sets]
        n_bits = np.array([int(np.log2(len(p))) for p in probs], np.int32)
        set_len = np.array([len(s) for s in sets], np.int32)
        set_cols = np.concatenate([np.asarray(s, np.int32) for s in sets])
        np.savez_compressed(OUT / f"noise_{name}.npz", probs=np.concatenate(probs), n_bits=n_bits,
                            transform=T, set_len=set_len, set_cols=set_cols,
                            exact=np.asarray(exact), ref_freq=np.asarray(freq),
                            ref_shots=np.int64(200_000))
        print(name, len(probs), "channels,", num_f, "f bits,", len(sets), "parity sets")


if __name__ == "__main__":
    main()
