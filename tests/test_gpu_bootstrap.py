"""Bootstrap replicates on the device (rnj_bootstrap): replicate r takes column
cols[r, k] of the original as its column k (dataloader::sample_fast_dist,
dataloader.cpp:16-58).  Each replicate's matrix must be bit-identical to the
plain call on the alignment resampled on the host."""
import ctypes
import ctypes.util

import numpy as np
import pytest

from oracle import oracle
from rapidnj_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def plain(ctx, seqs, typ, model, fastdist=True):
    aln = ctx.alignment(seqs, typ, fastdist=fastdist)
    mat = ctx.distance(aln, model)
    out, mx = mat.to_numpy(), mat.max
    mat.close()
    aln.close()
    return out, mx


def ulp_diff(a, b):
    a = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def check_replicates(ctx, seqs, typ, model, cols, fastdist=True, which=None, vs_oracle=2):
    """Every checked replicate equals the plain call on the host-resampled
    alignment bit for bit; the first `vs_oracle` of them also equal the oracle's
    matrix of that alignment (counts and transform restated from the reference,
    the same <= 1 ulp rule as the other parity tests)."""
    d = torch.from_numpy(seqs).cuda()
    outs, mx = ctx.bootstrap(d, cols, typ, model, fastdist=fastdist)
    for k, r in enumerate(range(cols.shape[0]) if which is None else which):
        rep = np.ascontiguousarray(seqs[:, cols[r]])
        want, wmx = plain(ctx, rep, typ, model, fastdist)
        got = outs[r].cpu().numpy()
        assert np.array_equal(got.view(np.int32), want.view(np.int32)), f"replicate {r}"
        assert mx[r] == np.float32(wmx)
        if k < vs_oracle:
            c = oracle.counts(rep, typ, naive=not fastdist, threads=8)
            ref, rmx = oracle.matrix(c, rep.shape[1], typ, oracle.JC if model == "jc" else
                                     oracle.KIMURA, naive=not fastdist)
            dd = ulp_diff(got, ref)
            assert dd.max() <= 1 and (dd == 1).sum() <= 2, f"replicate {r} vs the oracle"


@pytest.mark.parametrize("typ,model,fastdist", [(0, "kim", True), (0, "jc", True),
                                                (1, "kim", True), (0, "kim", False)])
def test_replicates_equal_host_resampling(ctx, typ, model, fastdist):
    rng = np.random.default_rng(typ * 10 + fastdist)
    seqs = (synth.tree_dna(300, 703, seed=4, mean_branch=0.05) if typ == 0
            else synth.tree_protein(300, 703, seed=4, mean_branch=0.2))
    cols = rng.integers(0, 703, size=(7, 703))
    check_replicates(ctx, seqs, typ, model, cols, fastdist)


def test_replicates_with_rapidnj_rand_sequence(ctx):
    # The columns rapidNJ draws: srand(0), then rand() % L for every column of
    # every replicate in turn (the C library's generator of this process).
    libc = ctypes.CDLL(ctypes.util.find_library("c"))
    libc.srand(0)
    L, R = 500, 4
    cols = np.array([[libc.rand() % L for _ in range(L)] for _ in range(R)])
    seqs = synth.tree_dna(200, L, seed=8)
    check_replicates(ctx, seqs, 0, "kim", cols)


def test_replicates_in_several_batches(ctx):
    # 66 replicates of 4000 sequences: more tiles than one batch holds, so the
    # replicates run in two chunks.
    rng = np.random.default_rng(5)
    seqs = synth.tree_dna(4000, 256, seed=6)
    cols = rng.integers(0, 256, size=(66, 256))
    check_replicates(ctx, seqs, 0, "kim", cols, which=(0, 61, 62, 65))


def test_rejects_bad_columns(ctx):
    from rapidnj_b200._native import RnjError
    seqs = synth.tree_dna(50, 100, seed=1)
    d = torch.from_numpy(seqs).cuda()
    with pytest.raises(RnjError):
        ctx.bootstrap(d, np.full((2, 100), 100), 0, "kim")
