"""The oracle's double-precision matrix (orc_matrix_d: each pair's value before
the reference's float cast, post-processed in double) against its float matrix
(orc_matrix, pinned to the reference's goldens): rounding every double entry
to float gives the float matrix bit for bit, for every model, alphabet, rule
set and the saturated cases (the maximum of the doubles rounds to the maximum
of the floats, and 2 x max scales exactly)."""
import numpy as np
import pytest

from oracle import oracle


def alignment(kind, n, L, seed):
    rng = np.random.default_rng(seed)
    if kind == "dna":
        a = np.frombuffer(b"ACGT-", np.uint8)[rng.integers(0, 5, (n, L))]
        return a, oracle.DNA
    if kind == "dna-related":
        root = rng.integers(0, 4, L)
        s = np.repeat(root[None, :], n, 0)
        m = rng.random((n, L)) < 0.15
        s[m] = rng.integers(0, 4, int(m.sum()))
        a = np.frombuffer(b"ACGT", np.uint8)[s]
        a[rng.random((n, L)) < 0.03] = ord("-")
        return a, oracle.DNA
    a = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY-", np.uint8)[rng.integers(0, 21, (n, L))]
    return a, oracle.PROTEIN


@pytest.mark.parametrize("kind", ["dna", "dna-related", "protein"])
@pytest.mark.parametrize("model", [oracle.JC, oracle.KIMURA])
@pytest.mark.parametrize("naive", [False, True])
def test_double_matrix_rounds_to_the_float_matrix(kind, model, naive):
    seqs, typ = alignment(kind, 60, 97, seed=3)
    c = oracle.counts(seqs, typ, naive=naive)
    want, wmax = oracle.matrix(c, seqs.shape[1], typ, model, naive=naive)
    got, gmax = oracle.matrix_f64(c, seqs.shape[1], typ, model, naive=naive)
    assert np.array_equal(got.astype(np.float32).view(np.int32), want.view(np.int32))
    assert np.float32(gmax) == np.float32(wmax)
    assert (np.diag(got) == 0).all() and np.array_equal(got, got.T)


def test_double_values_of_single_pairs():
    lib = oracle.lib()
    # K2P: -0.5 log(1 - 2 ts - tv) - 0.25 log(1 - 2 tv) from the float quotients
    ts, tv = np.float32(10 / 100), np.float32(5 / 100)
    want = -0.5 * np.log(1.0 - 2.0 * float(ts) - float(tv)) - 0.25 * np.log(1.0 - 2.0 * float(tv))
    assert abs(lib.orc_k2p_d(10, 5, 100) - want) <= 2e-16 * abs(want)
    assert lib.orc_k2p_d(1, 1, 0) == -1.0 and lib.orc_k2p_d(40, 30, 100) == -1.0
    # JC: valid 0 gives -0.0; saturation -1
    assert lib.orc_jc_d(0, 0, 0, oracle.DNA) == 0.0 and lib.orc_jc_d(3, 0, 4, oracle.DNA) == -1.0
    # protein: the Dayhoff table and the 10.0 cap keep their double values
    assert lib.orc_kimura_protein_d(80, 100) == lib.orc_pam_value(50) / 100.0
    assert lib.orc_kimura_protein_d(95, 100) == 10.0
