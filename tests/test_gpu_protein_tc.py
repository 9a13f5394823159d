"""Protein on the tensor cores: FP4 features [valid | one-hot residue rank ...],
two f32 accumulators (V = both residues, M = same residue), mismatches = V - M.
The counts must equal the bit-plane kernel's (RNJ_POPCOUNT) bit for bit, and
so must every distance computed from them; alphabets of more than 31 residues
fall back to the bit planes."""
import numpy as np
import pytest

from oracle import oracle
from rapidnj_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

# 31 distinct residue bytes (case matters; b/B/J/j/x/X/z/Z/? and . - are gaps)
RES31 = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWYOUacdefghik", dtype=np.uint8)
RES32 = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWYOUacdefghikl", dtype=np.uint8)


def alignment(n, L, alphabet, gap=0.06, seed=0):
    rng = np.random.default_rng(seed)
    root = alphabet[rng.integers(0, alphabet.size, L)]
    seqs = np.repeat(root[None, :], n, axis=0)
    mut = rng.random((n, L)) < 0.25
    seqs[mut] = alphabet[rng.integers(0, alphabet.size, int(mut.sum()))]
    seqs[rng.random((n, L)) < gap] = ord("-")
    seqs[:, 0] = alphabet[0]  # a residue in the first column of every row
    return np.ascontiguousarray(seqs)


def counts(ctx, seqs, popcount):
    aln = ctx.alignment(seqs, 1, popcount=popcount)
    n = seqs.shape[0]
    out = torch.zeros(n * n * 3, dtype=torch.int32, device="cuda")
    ctx.counts_into(aln, out)
    aln.close()
    return out.cpu().numpy().view(np.uint32).reshape(n, n, 3)


def matrix(ctx, seqs, model, popcount, compat_wrap=False):
    aln = ctx.alignment(seqs, 1, popcount=popcount, compat_wrap=compat_wrap)
    mat = ctx.distance(aln, model)
    out, mx = mat.to_numpy(), mat.max
    mat.close()
    aln.close()
    return out, mx


@pytest.mark.parametrize("n,L", [(2, 1), (40, 31), (130, 32), (129, 33), (200, 255), (257, 256),
                                 (300, 257), (128, 1024), (500, 1500), (1000, 700)])
def test_counts_equal_bit_planes(ctx, n, L):
    seqs = synth.tree_protein(n, L, seed=n * 7 + L, mean_branch=0.2)
    assert np.array_equal(counts(ctx, seqs, False), counts(ctx, seqs, True))


@pytest.mark.parametrize("alphabet", [RES31[:2], RES31[:5], RES31[:20], RES31, RES32])
def test_alphabet_sizes(ctx, alphabet):
    seqs = alignment(300, 600, alphabet, seed=alphabet.size)
    assert np.array_equal(counts(ctx, seqs, False), counts(ctx, seqs, True))
    for model in ("kim", "jc"):
        a, ma = matrix(ctx, seqs, model, False)
        b, mb = matrix(ctx, seqs, model, True)
        assert np.array_equal(a.view(np.int32), b.view(np.int32)) and ma == mb


@pytest.mark.parametrize("L", [128, 384, 1000])
@pytest.mark.parametrize("compat_wrap", [False, True])
def test_distances_equal_bit_planes(ctx, L, compat_wrap):
    seqs = synth.tree_protein(400, L, seed=L, mean_branch=0.3)
    for model in ("kim", "jc"):
        a, ma = matrix(ctx, seqs, model, False, compat_wrap)
        b, mb = matrix(ctx, seqs, model, True, compat_wrap)
        assert np.array_equal(a.view(np.int32), b.view(np.int32)) and ma == mb


def test_against_oracle(ctx):
    seqs = synth.tree_protein(250, 900, seed=3, mean_branch=0.4)
    c = counts(ctx, seqs, False)
    assert np.array_equal(c, oracle.counts(seqs, oracle.PROTEIN))
    got, mx = matrix(ctx, seqs, "kim", False)
    ref, rmx = oracle.matrix(c, seqs.shape[1], oracle.PROTEIN, oracle.KIMURA)
    d = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert d.max() <= 1 and (d == 1).sum() <= 2
