"""Shards on the GPU: an alignment's tiles split into 1..5 shards, all run on one
device one after another (each shard's kernels are independent of the others'),
the maximum exchanged on the host, and the shards' host copies assembled.  The
result must equal the one-call matrix bit for bit, on every kernel family."""
import numpy as np
import pytest

import oracle.oracle as O

pytestmark = pytest.mark.gpu


def assemble(ctx, aln, model, nshards, full=False):
    from rapidnj_b200 import api
    n = aln.n
    shards = [api.Shard(ctx, aln, model, s, nshards) for s in range(nshards)]
    g = max(sh.run() for sh in shards)
    host = np.full((n, n), np.nan, np.float32)
    copied = 0
    for sh in shards:
        sh.finish(g)
        copied += sh.copy_tiles(host)
    if full:
        assert copied == n * n * 4
        out = host
    else:
        out = np.triu(host) + np.triu(host, 1).T
    return out, g, shards


def saturating_dna(n, L, seed):
    rng = np.random.default_rng(seed)
    s = rng.choice(np.frombuffer(b"ACGT-", np.uint8), size=(n, L), p=[0.24] * 4 + [0.04])
    s[3, :] = ord("-")
    return s


CASES = [
    ("dna-k2p-tc", lambda: saturating_dna(700, 40, 1), O.DNA, "kim", {}),
    ("dna-jc-tc", lambda: saturating_dna(300, 30, 2), O.DNA, "jc", {}),
    ("dna-k2p-popcount", lambda: saturating_dna(520, 300, 3), O.DNA, "kim", {"popcount": True}),
    ("dna-tree-tc", None, O.DNA, "kim", {}),
    ("protein-kimura", None, O.PROTEIN, "kim", {}),
    ("dna-naive-full", lambda: saturating_dna(400, 64, 4), O.DNA, "kim",
     {"fastdist": False, "full_rows": True}),
]


@pytest.mark.parametrize("name,make,type_,model,kw", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("nshards", [1, 2, 3, 5])
def test_shards_assemble_the_one_call_matrix(ctx, name, make, type_, model, kw, nshards):
    from rapidnj_b200 import synth
    if name == "dna-tree-tc":
        seqs = synth.tree_dna(650, 1200, seed=7)
    elif name == "protein-kimura":
        seqs = synth.tree_protein(450, 500, seed=8)
    else:
        seqs = make()
    aln = ctx.alignment(seqs, type_, **kw)
    want = ctx.distance(aln, model)
    ref = want.to_numpy()
    got, g, shards = assemble(ctx, aln, model, nshards, kw.get("full_rows", False))
    assert g == want.max
    assert np.array_equal(got, ref)
    for sh in shards:
        sh.close()


def test_shard_matches_oracle_and_device_output(ctx):
    """One shard of two, checked against the oracle on its own tiles (device copy,
    mirrors included)."""
    import torch
    from rapidnj_b200 import api
    seqs = saturating_dna(333, 50, 9)
    want, mx = O.distance_matrix(seqs, O.KIMURA, O.DNA)
    aln = ctx.alignment(seqs, O.DNA)
    out = torch.full((333, 340), 5.0, dtype=torch.float32, device="cuda")
    sh0 = api.Shard(ctx, aln, "kim", 0, 2)
    sh1 = api.Shard(ctx, aln, "kim", 1, 2, out=out)
    g = max(sh0.run(), sh1.run())
    assert g == mx
    sh1.finish(g)
    dev = out.cpu().numpy()
    t0, t1, _ = api.shard_tiles(333, 1, 2)
    for t in range(t0, t1):
        ti, tj = api.tile_coords(333, t)
        r, c = slice(ti * 128, min(333, ti * 128 + 128)), slice(tj * 128, min(333, tj * 128 + 128))
        assert np.array_equal(dev[r, c], want[r, c])
        assert np.array_equal(dev[c, r], want[c, r])
    assert (dev[:, 333:] == 5.0).all()


def test_sharded_distance_single_process(ctx):
    from rapidnj_b200 import sharded
    seqs = saturating_dna(260, 40, 10)
    aln = ctx.alignment(seqs, O.DNA)
    sh, g = sharded.sharded_distance(ctx, aln, "kim")
    host = np.zeros((260, 260), np.float32)
    sh.copy_tiles(host)
    want, mx = O.distance_matrix(seqs, O.KIMURA, O.DNA)
    assert g == mx
    assert np.array_equal(np.triu(host) + np.triu(host, 1).T, want)
