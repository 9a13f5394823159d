"""Seeded synthetic alignments with the shapes and value distributions of the
benchmark workloads (no public dataset exists for this path; every input is
generated here).

Workloads
---------
* ``iid_dna``      uniform i.i.d. A/C/G/T, each cell independently '-' with
                   probability ``gap`` (the 512 x 2,000 Jukes-Cantor case).
* ``tree_dna``     a uniform random root evolved down a random binary tree
                   (Yule process: a uniformly chosen leaf splits at each step),
                   branch lengths ~ Exp(mean), Kimura-2P substitution with
                   transition/transversion ratio R = alpha / (2 beta) = 2
                   (kappa = alpha / beta = 4), then uniform random gaps
                   (the 10,000 x 10,000 and 50,000 x 1,000 Kimura-2P cases).
* ``tree_protein`` the same tree process over the 20 amino acids with
                   equal-rate (Poisson) substitution, then gaps placed in runs
                   of geometric length (mean 3) until the gap fraction is
                   reached (the 5,000 x 1,500 protein Kimura case).
* ``batch_mix``    the 256-alignment batch: N ~ U[32, 2048], L ~ U[300, 5000],
                   70 % tree DNA, 30 % tree protein.
* ``served_stream`` request sizes of the served workload: N log-uniform in
                   [16, 4096], L log-uniform in [200, 8000], 50/50 DNA
                   Jukes-Cantor / protein Kimura.

Sequences are returned as an ``(n, L)`` ``uint8`` array of ASCII bytes.
"""
from __future__ import annotations

import numpy as np

DNA_LETTERS = np.frombuffer(b"AGTC", dtype=np.uint8)  # code 0..3: A, G, T, C
AMINO = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", dtype=np.uint8)
GAP = ord("-")


def iid_dna(n: int, L: int, gap: float = 0.05, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    codes = rng.integers(0, 4, size=(n, L), dtype=np.uint8)
    seqs = DNA_LETTERS[codes]
    if gap > 0:
        seqs[rng.random((n, L), dtype=np.float32) < gap] = GAP
    return seqs


def iid_protein(n: int, L: int, gap: float = 0.05, seed: int = 0) -> np.ndarray:
    """Uniform i.i.d. amino acids, each cell '-' with probability ``gap``."""
    rng = np.random.default_rng(seed)
    seqs = AMINO[rng.integers(0, AMINO.size, size=(n, L), dtype=np.uint8)]
    if gap > 0:
        seqs[rng.random((n, L), dtype=np.float32) < gap] = GAP
    return seqs


def _k2p_probs(t: float, kappa: float) -> tuple[float, float]:
    """Per-site transition and (total) transversion probabilities after a
    branch of t substitutions per site (rate normalised to alpha + 2 beta = 1)."""
    beta = 1.0 / (kappa + 2.0)
    alpha = kappa * beta
    e1 = np.exp(-4.0 * beta * t)
    e2 = np.exp(-2.0 * (alpha + beta) * t)
    p_ts = 0.25 + 0.25 * e1 - 0.5 * e2
    p_tv = 0.5 - 0.5 * e1
    return float(p_ts), float(p_tv)


def _mutate_positions(rng, L: int, p: float) -> np.ndarray:
    k = rng.binomial(L, min(max(p, 0.0), 1.0))
    if k == 0:
        return np.empty(0, dtype=np.int64)
    if k > L // 8:
        return np.flatnonzero(rng.random(L) < p)
    return np.unique(rng.integers(0, L, size=k))


def _yule(n: int, L: int, root: np.ndarray, evolve, rng) -> np.ndarray:
    out = np.empty((n, L), dtype=np.uint8)
    out[0] = root
    for m in range(1, n):
        k = int(rng.integers(0, m))
        parent = out[k].copy()
        out[k] = evolve(parent)
        out[m] = evolve(parent)
    return out


def tree_dna(n: int, L: int, mean_branch: float = 0.02, ratio: float = 2.0,
             gap: float = 0.03, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    kappa = 2.0 * ratio

    def evolve(parent: np.ndarray) -> np.ndarray:
        child = parent.copy()
        t = rng.exponential(mean_branch)
        p_ts, p_tv = _k2p_probs(t, kappa)
        pos = _mutate_positions(rng, L, p_ts + p_tv)
        if pos.size:
            u = rng.random(pos.size) * (p_ts + p_tv)
            xor = np.where(u < p_ts, 1, np.where(u < p_ts + 0.5 * p_tv, 2, 3)).astype(np.uint8)
            child[pos] ^= xor
        return child

    root = rng.integers(0, 4, size=L, dtype=np.uint8)
    seqs = DNA_LETTERS[_yule(n, L, root, evolve, rng)]
    if gap > 0:
        seqs[rng.random((n, L), dtype=np.float32) < gap] = GAP
    return seqs


def _geometric_gap_runs(seqs: np.ndarray, frac: float, mean_run: float, rng) -> None:
    n, L = seqs.shape
    target = int(frac * n * L)
    placed = 0
    p = 1.0 / mean_run
    while placed < target:
        batch = max(1, (target - placed) // int(mean_run))
        rows = rng.integers(0, n, size=batch)
        starts = rng.integers(0, L, size=batch)
        lens = rng.geometric(p, size=batch)
        for r, s, ln in zip(rows, starts, lens):
            e = min(L, s + ln)
            seqs[r, s:e] = GAP
            placed += e - s
            if placed >= target:
                break


def tree_protein(n: int, L: int, mean_branch: float = 0.05, gap: float = 0.08,
                 mean_gap_run: float = 3.0, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    A = AMINO.size

    def evolve(parent: np.ndarray) -> np.ndarray:
        child = parent.copy()
        t = rng.exponential(mean_branch)
        p = (A - 1) / A * (1.0 - np.exp(-A / (A - 1) * t))
        pos = _mutate_positions(rng, L, p)
        if pos.size:
            shift = rng.integers(1, A, size=pos.size, dtype=np.uint8)
            child[pos] = (child[pos] + shift) % A
        return child

    root = rng.integers(0, A, size=L, dtype=np.uint8)
    seqs = AMINO[_yule(n, L, root, evolve, rng)]
    if gap > 0:
        _geometric_gap_runs(seqs, gap, mean_gap_run, rng)
    return seqs


def batch_mix(count: int = 256, seed: int = 0, n_range=(32, 2048), l_range=(300, 5000),
              dna_frac: float = 0.7):
    """List of (kind, seqs) for the batched workload; kind is 'dna' or 'protein'."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        L = int(rng.integers(l_range[0], l_range[1] + 1))
        if rng.random() < dna_frac:
            out.append(("dna", tree_dna(n, L, seed=seed * 100003 + k)))
        else:
            out.append(("protein", tree_protein(n, L, seed=seed * 100003 + k)))
    return out


def served_sizes(count: int, seed: int = 0, n_range=(16, 4096), l_range=(200, 8000)):
    """(kind, n, L) triples of the served workload: log-uniform sizes, 50/50 DNA
    Jukes-Cantor / protein Kimura."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(round(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1])))))
        L = int(round(np.exp(rng.uniform(np.log(l_range[0]), np.log(l_range[1])))))
        out.append(("dna" if rng.random() < 0.5 else "protein", n, L))
    return out


def write_fasta(path: str, seqs: np.ndarray, names=None, width: int = 0) -> None:
    n, L = seqs.shape
    with open(path, "wb") as f:
        for i in range(n):
            name = names[i] if names is not None else f"s{i}"
            f.write(b">" + name.encode() + b"\n")
            row = seqs[i].tobytes()
            if width:
                for s in range(0, L, width):
                    f.write(row[s:s + width] + b"\n")
            else:
                f.write(row + b"\n")
