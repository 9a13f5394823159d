"""Generates tests/golden/nj_*.npz: the reference's own neighbour-joining set-up
(rapidNJ::initialize, rapidNJ.cpp:94-141; rapidNJMem::initialize,
rapidNJMem.cpp:92-135) over distance matrices, through oracle/_ref/nj_harness
(compiled from the reference sources by oracle/Makefile).

Runs only where the rapidNJ source tree is present; the outputs are committed and
the tests only read them.

Matrices
--------
* the reference's own matrices of its fixtures (tests/golden/fixture_*.npz):
  LGT_70 K2P and JC, PF15224 Kimura;
* the crafted DNA case at L = 64 (identical rows, saturated pairs);
* tree-evolved DNA with classes of identical sequences (sizes 2, 3 and 5; K2P
  gives -0 between identical sequences), K2P, by the oracle (bit-identical to
  the reference's drivers);
* unrelated random DNA (most pairs saturated: many equal distances), K2P;
* 40 identical sequences (every row redundant but the last);
* n = 1, 2 and 3.

For each matrix and cap in {0 (rapidNJ), 5 (rapidNJMem, sortedMatrixSize 5)}:
separation sums, separations, maxRowSeparations, max_separation, indexToId,
redundantToMasterMap, redundantCount, row_lengths, the redundantMap lists
(lengths + concatenation) and the sorted rows (ids + distances, concatenated).

Usage: python tests/golden/make_golden_nj.py   (from the repository root)
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402  (test infrastructure)
from rapidnj_b200 import synth  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")
CAPS = (0, 5)


def k2p(seqs):
    m, _ = oracle.distance_matrix(seqs, oracle.KIMURA, oracle.DNA)
    return m


def matrices():
    out = {}
    z = np.load(os.path.join(OUT, "fixture_LGT_70.npz"))
    out["lgt70_kim"] = z["kim_fast"]
    out["lgt70_jc"] = z["jc_fast"]
    out["pf15224_kim"] = np.load(os.path.join(OUT, "fixture_PF15224_full.npz"))["kim_fast"]
    out["crafted_dna_L64"] = np.load(os.path.join(OUT, "dna_L64.npz"))["kim_fast"]
    s = synth.tree_dna(150, 300, seed=31, mean_branch=0.05)
    for dst, src in ((4, 90), (17, 90), (60, 33), (100, 12), (101, 12), (120, 12), (149, 12)):
        s[dst] = s[src]
    out["tree_classes"] = k2p(s)
    out["saturated"] = k2p(synth.iid_dna(120, 40, gap=0.0, seed=7))
    out["identical"] = k2p(np.repeat(synth.iid_dna(1, 80, gap=0.0, seed=3), 40, axis=0))
    for n in (1, 2, 3):
        out[f"n{n}"] = k2p(synth.tree_dna(n, 50, seed=n, mean_branch=0.1))
    return out


def main():
    if not os.path.exists(os.path.join(oracle.REF_DIR, "nj_harness")):
        raise SystemExit("oracle/_ref/nj_harness is not built (make -C oracle ref)")
    for name, m in matrices().items():
        m = np.ascontiguousarray(m, dtype=np.float32)
        d = {"matrix": m}
        for cap in CAPS:
            r, _ = oracle.ref_nj_init(m, cap)
            p = f"c{cap}_"
            for k in ("sums", "separations", "max_row_separations", "index_to_id",
                      "redundant_to_master", "redundant_count", "row_lengths"):
                d[p + k] = r[k]
            d[p + "max_separation"] = np.float32(r["max_separation"])
            d[p + "list_len"] = np.array([len(x) for x in r["lists"]], dtype=np.int32)
            d[p + "list_cat"] = np.array([v for x in r["lists"] for v in x], dtype=np.int32)
            ids = [x[0] for x in r["rows"] if x is not None]
            dist = [x[1] for x in r["rows"] if x is not None]
            d[p + "row_ids"] = np.concatenate(ids) if ids else np.zeros(0, np.uint32)
            d[p + "row_dist"] = np.concatenate(dist) if dist else np.zeros(0, np.float32)
        np.savez_compressed(os.path.join(OUT, f"nj_{name}.npz"), **d)
        print(name, m.shape)


if __name__ == "__main__":
    main()
