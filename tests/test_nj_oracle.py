"""The NJ set-up restatement (oracle.nj_init) against the reference's own
rapidNJ::initialize / rapidNJMem::initialize results committed under
tests/golden/nj_*.npz (made by tests/golden/make_golden_nj.py)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle
from njcheck import compare, golden

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "nj_*.npz")))


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[3:-4] for p in GOLDEN])
@pytest.mark.parametrize("cap", [0, 5])
def test_oracle_matches_reference(path, cap):
    z = np.load(path)
    got = oracle.nj_init(z["matrix"], cap)
    compare(got, golden(z, cap), cap, exact_ties=False)


def test_goldens_present():
    assert len(GOLDEN) >= 10


def test_golden_cases_cover_redundancy_and_ties():
    # the fixtures hold redundant rows (classes of 2, 3 and 5) and equal distances
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "nj_tree_classes.npz"))
    g = golden(z, 0)
    assert sorted(set(g["redundant_count"].tolist())) == [1, 2, 3, 5]
    s = np.load(os.path.join(os.path.dirname(__file__), "golden", "nj_saturated.npz"))
    d = golden(s, 0)["rows"][-1][1]
    assert len(np.unique(d)) < len(d)
    i = np.load(os.path.join(os.path.dirname(__file__), "golden", "nj_identical.npz"))
    assert (golden(i, 0)["index_to_id"] == -1).sum() == 39


@pytest.mark.skipif(not os.path.exists(os.path.join(oracle.REF_DIR, "nj_harness")),
                    reason="the reference harness is not built here")
def test_oracle_matches_reference_live():
    from rapidnj_b200 import synth
    s = synth.tree_dna(90, 200, seed=4, mean_branch=0.04)
    s[3] = s[70]
    m, _ = oracle.distance_matrix(s, oracle.JC, oracle.DNA)
    for cap in (0, 9):
        want, _ = oracle.ref_nj_init(m, cap)
        compare(oracle.nj_init(m, cap), want, cap, exact_ties=False)
