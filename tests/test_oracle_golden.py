"""The CPU oracle against the reference's own outputs (golden vectors).

Every golden was produced by the reference itself (tests/golden/make_golden.py);
passing here pins the oracle, which the GPU parity tests then use at sizes and
shapes the goldens do not cover.
"""
import numpy as np
import pytest

from conftest import golden_files, golden_type, load_golden
from oracle import oracle

GOLDENS = golden_files()


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def wrap_fast_protein(c, L):
    """The reference fast protein estimator's valid count, as its uint32 dump holds it."""
    lib = oracle.lib()
    out = c.copy()
    n = c.shape[0]
    iu = np.triu_indices(n, 1)
    v = [lib.orc_protein_fast_valid(int(x), L) & 0xFFFFFFFF for x in c[..., 2][iu]]
    out[..., 2][iu] = np.array(v, dtype=np.uint32)
    return out


@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
def test_type_detection(path):
    g = load_golden(path)
    if g["type_arg"] == "auto":
        assert oracle.detect_type(g["chars"]) == int(g["ref_type"])


@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
def test_counts(path):
    g = load_golden(path)
    seqs, typ = g["chars"], golden_type(g)
    L = seqs.shape[1]
    fast = oracle.counts(seqs, typ, naive=False)
    if typ == oracle.PROTEIN and L % 128 == 0:
        fast = wrap_fast_protein(fast, L)
    assert np.array_equal(fast, g["counts_fast"])
    assert np.array_equal(oracle.counts(seqs, typ, naive=True), g["counts_naive"])
    assert np.array_equal(oracle.counts(seqs, typ, naive=True, full=True), g["counts_naive_full"])


@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
@pytest.mark.parametrize("model,mk", [(oracle.JC, "jc"), (oracle.KIMURA, "kim")])
@pytest.mark.parametrize("naive", [False, True])
def test_matrices(path, model, mk, naive):
    g = load_golden(path)
    seqs, typ = g["chars"], golden_type(g)
    c = oracle.counts(seqs, typ, naive)
    m, _ = oracle.matrix(c, seqs.shape[1], typ, model, naive,
                         compat_wrap=(typ == oracle.PROTEIN and not naive))
    ref = g[f"{mk}_{'naive' if naive else 'fast'}"]
    assert np.array_equal(bits(m), bits(ref))


@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
def test_disk_rows(path):
    g = load_golden(path)
    seqs, typ = g["chars"], golden_type(g)
    L = seqs.shape[1]
    m, _ = oracle.matrix(oracle.counts(seqs, typ, False), L, typ, oracle.KIMURA, False,
                         compat_wrap=(typ == oracle.PROTEIN))
    assert np.array_equal(bits(m), bits(g["kim_fast_disk"]))
    cf = oracle.counts(seqs, typ, True, full=True)
    mf, _ = oracle.matrix(cf, L, typ, oracle.KIMURA, True, full=True)
    assert np.array_equal(bits(mf), bits(g["kim_naive_disk"]))


def test_pam_table_walk_covers_range():
    g = load_golden(f"{oracle.HERE}/../tests/golden/protein_pam_walk.npz")
    m = g["kim_fast"]
    # pairs (0, k) walk p from 0.70 to 1.00: 10.0 above 0.93, table values between
    row = m[0, 1:]
    assert (row == 10.0).any()
    assert ((row > 1.9) & (row < 10.0)).sum() > 20


def test_planted_error_is_caught():
    """A mistake planted in the oracle's output must be visible to the check."""
    g = load_golden(f"{oracle.HERE}/../tests/golden/fixture_LGT_70.npz")
    c = oracle.counts(g["chars"], oracle.DNA)
    c[0, 1, 0] += 1
    assert not np.array_equal(c, g["counts_fast"])
