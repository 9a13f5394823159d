"""Autotuned launch choices change the time of a distance call, never its
result: every choice (tensor cores or bit planes for DNA, a K split of the
bit-plane kernel, the tile-order band and transform occupancy of the
tensor-core kernel, the streamed call's band height) gives the same bits as
the defaults, and rnj_tune stores a choice that the next calls use."""
import numpy as np
import pytest

from rapidnj_b200 import api, synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(autouse=True)
def empty_table():
    api.tune_clear()
    yield
    api.tune_clear()


def device_matrix(ctx, seqs, typ, model):
    aln = ctx.alignment(seqs, typ)
    mat = ctx.distance(aln, model)
    out, mx = mat.to_numpy(), mat.max
    mat.close()
    aln.close()
    return out, mx


def same(a, b):
    assert np.array_equal(a[0].view(np.int32), b[0].view(np.int32)) and a[1] == b[1]


@pytest.mark.parametrize("fields", [
    dict(dna_kernel=1),
    dict(dna_kernel=1, ksplit=4),
    dict(tile_band=4, transform_ctas=3),
    dict(tile_band=1, transform_ctas=1),
    dict(tc_stages=2),
    dict(tc_stages=4, tile_band=8),
    dict(tc_epilogue=1, tc_stages=5),
    dict(tc_epilogue=1, tc_stages=2, transform_ctas=2),
    dict(dna_kernel=1, pop_stages=3),
    dict(dna_kernel=1, pop_stages=2, ksplit=2),
])
@pytest.mark.parametrize("model", ["kim", "jc"])
def test_dna_choices_give_default_bits(ctx, fields, model):
    seqs = synth.tree_dna(700, 3000, seed=4, mean_branch=0.05)
    ref = device_matrix(ctx, seqs, 0, model)
    api.tune_set(700, 3000, "dna", **fields)
    same(device_matrix(ctx, seqs, 0, model), ref)


@pytest.mark.parametrize("fields", [dict(ksplit=2), dict(ksplit=3), dict(ksplit=8),
                                    dict(ksplit=16), dict(pop_stages=2), dict(pop_stages=3),
                                    dict(ksplit=4, pop_stages=2)])
def test_protein_bit_plane_choices_give_default_bits(ctx, fields):
    seqs = synth.tree_protein(300, 2500, seed=6, mean_branch=0.2)
    ref = device_matrix(ctx, seqs, 1, "kim")
    api.tune_set(300, 2500, "protein", dna_kernel=1, **fields)
    same(device_matrix(ctx, seqs, 1, "kim"), ref)


@pytest.mark.parametrize("stages", [2, 3, 6])
def test_protein_tensor_core_ring_depth_gives_default_bits(ctx, stages):
    seqs = synth.tree_protein(400, 1500, seed=8, mean_branch=0.1)
    ref = device_matrix(ctx, seqs, 1, "kim")
    api.tune_set(400, 1500, "protein", tc_stages=stages)
    same(device_matrix(ctx, seqs, 1, "kim"), ref)


def test_batch_takes_its_shape_from_the_tuner(ctx):
    # Two alignments; the larger one's bucket is tuned to a three-stage ring
    # and band 4: the batch re-captures its graph with that ring depth, and the
    # results equal the untuned batch's.
    dna = synth.tree_dna(900, 2000, seed=2)
    prot = synth.tree_protein(200, 700, seed=3)

    def run():
        b = api.Batch(ctx, max_alignments=4, max_tiles=4096)
        slots = [b.add(ctx.alignment(dna, 0), "kim"), b.add(ctx.alignment(prot, 1), "kim")]
        b.run()
        b.synchronize()
        out = []
        for k in slots:
            m = b.take(k)
            out.append((m.to_numpy(), m.max))
            m.close()
        shape = b.tuning()
        b.close()
        return out, shape

    ref, shape0 = run()
    assert shape0 == (6, 0)
    api.tune_set(900, 2000, "dna", tc_stages=3, tile_band=4)
    got, shape1 = run()
    assert shape1 == (3, 1)
    for g, r in zip(got, ref):
        same(g, r)


def test_stream_band_gives_default_bits(ctx):
    seqs = synth.tree_dna(1500, 1200, seed=9)
    out = torch.empty((1500, 1500), dtype=torch.float32).pin_memory().numpy()
    ref = ctx.distance_matrix_host(seqs, "kim", "dna", band_tiles=-1)
    for band in (2, 5):
        api.tune_set(1500, 1200, "dna", stream_band=band)
        got = ctx.distance_matrix_host(seqs, "kim", "dna", out=out)
        same(got, ref)


@pytest.mark.parametrize("n,L,typ", [(600, 4000, "dna"), (260, 3000, "protein")])
def test_tune_stores_a_choice_that_later_calls_use(ctx, n, L, typ):
    p = ctx.tune(n, L, typ)
    assert p.ms > 0
    got = api.tune_get(n, L, typ)
    assert got is not None and got.as_dict() == p.as_dict()
    # the tuned bucket computes the same distances as the defaults
    seqs = synth.tree_dna(n, L, seed=1) if typ == "dna" else synth.tree_protein(n, L, seed=1)
    t = 0 if typ == "dna" else 1
    tuned = device_matrix(ctx, seqs, t, "kim")
    api.tune_clear()
    same(tuned, device_matrix(ctx, seqs, t, "kim"))


def test_k_split_helps_few_long_sequences(ctx):
    # 256 protein sequences x 20,000 columns on the bit planes: 3 triangle
    # tiles, so one CTA per tile uses 3 of 148 SMs; the tuner must find that
    # splitting the columns is faster.
    p = ctx.tune(256, 20000, "protein", popcount=True)
    assert p.ksplit > 1
