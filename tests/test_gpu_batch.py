"""The batched form: many alignments of uneven size and kind in one persistent,
graph-captured pass give exactly the matrices of one plain call per alignment."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def mixed_set(seed=0, count=24):
    from rapidnj_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(2, 400))
        L = int(rng.integers(1, 3000))
        r = k % 6
        if r == 0:
            out.append((synth.tree_dna(n, L, seed=k, mean_branch=0.1), 0, "kim", {}))
        elif r == 1:
            out.append((synth.iid_dna(n, L, seed=k), 0, "jc", {}))
        elif r == 2:
            out.append((synth.tree_protein(n, L, seed=k), 1, "kim", {}))
        elif r == 3:
            out.append((synth.tree_protein(n, L, seed=k), 1, "jc", {}))
        elif r == 4:
            out.append((synth.tree_dna(n, L, seed=k), 0, "kim", {"popcount": True}))
        else:
            s = synth.tree_dna(n, L, seed=k, mean_branch=0.2)
            s[rng.random(s.shape) < 0.02] = ord("u")
            out.append((s, 0, "kim", {"fastdist": False}))
    return out


def test_batch_matches_plain_calls(ctx):
    from rapidnj_b200 import api
    items = mixed_set(0)
    batch = api.Batch(ctx, max_alignments=64, max_tiles=4096)
    alns, slots = [], []
    for seqs, typ, model, kw in items:
        a = ctx.alignment(seqs, typ, **kw)
        alns.append(a)
        slots.append(batch.add(a, model))
    batch.run()
    batch.synchronize()
    for (seqs, typ, model, kw), a, slot in zip(items, alns, slots):
        ref = ctx.distance(a, model)
        got = batch.take(slot)
        assert np.array_equal(got.to_numpy(), ref.to_numpy())
        assert got.max == ref.max
    batch.close()


def test_batch_graph_reused_across_runs(ctx):
    """A second run with other alignments (no re-capture) is still exact, and
    state of the first run (maxima, flags) does not leak into the second."""
    from rapidnj_b200 import api
    batch = api.Batch(ctx, max_alignments=64, max_tiles=4096)
    for seed in (1, 2):
        items = mixed_set(seed, count=12)
        outs, alns = [], []
        for seqs, typ, model, kw in items:
            a = ctx.alignment(seqs, typ, **kw)
            n = seqs.shape[0]
            o = torch.full((n, n + 2), 3.0, dtype=torch.float32, device="cuda")
            batch.add(a, model, out=o)
            outs.append(o)
            alns.append(a)
        batch.run()
        batch.synchronize()
        for (seqs, typ, model, kw), a, o in zip(items, alns, outs):
            n = seqs.shape[0]
            ref = ctx.distance(a, model).to_numpy()
            assert np.array_equal(o[:, :n].cpu().numpy(), ref)
            assert (o[:, n:] == 3.0).all()
        batch.clear()
    batch.close()


def test_batch_add_many_matches_plain(ctx):
    """Packing and adding many device alignments in one call (one alphabet
    synchronisation for all protein alignments) gives the plain matrices."""
    from rapidnj_b200 import api
    items = [it for it in mixed_set(5, count=18) if not it[3]]  # default flags only
    batch = api.Batch(ctx, max_alignments=32, max_tiles=2048)
    dev = [torch.from_numpy(s).cuda() for s, _, _, _ in items]
    slots = batch.add_many(dev, [t for _, t, _, _ in items], [m for _, _, m, _ in items])
    batch.run()
    for (seqs, typ, model, _), slot in zip(items, slots):
        ref = ctx.distance(ctx.alignment(seqs, typ), model).to_numpy()
        assert np.array_equal(batch.take(slot).to_numpy(), ref)
    batch.clear()
    assert batch.size() == (0, 0)
    batch.close()


def test_batch_against_oracle(ctx):
    from rapidnj_b200 import api, synth
    batch = api.Batch(ctx, max_alignments=8, max_tiles=256)
    cases = [(synth.tree_dna(300, 500, seed=3, mean_branch=0.2), oracle.DNA, "kim", oracle.KIMURA),
             (synth.tree_protein(200, 700, seed=4), oracle.PROTEIN, "kim", oracle.KIMURA)]
    slots = []
    for seqs, typ, model, _ in cases:
        slots.append(batch.add(ctx.alignment(seqs, typ), model))
    batch.run()
    for (seqs, typ, model, mo), slot in zip(cases, slots):
        ref, mx = oracle.matrix(oracle.counts(seqs, typ), seqs.shape[1], typ, mo)
        got = batch.take(slot).to_numpy()
        d = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
        assert d.max() <= 1 and (d == 1).sum() <= 2


def test_batch_capacity_errors(ctx):
    from rapidnj_b200 import api, synth, RnjError
    batch = api.Batch(ctx, max_alignments=2, max_tiles=3)
    a = ctx.alignment(synth.tree_dna(300, 100, seed=1), 0)  # 3 x 4 / 2 = 6 tiles
    with pytest.raises(RnjError, match="tiles"):
        batch.add(a, "kim")
    small = ctx.alignment(synth.tree_dna(10, 100, seed=1), 0)
    batch.add(small, "kim")
    batch.add(small, "jc")
    with pytest.raises(RnjError, match="alignments"):
        batch.add(small, "kim")
    assert batch.size() == (2, 2)
