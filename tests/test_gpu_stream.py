"""The streamed host-to-host call (rnj_distance_matrix_host[_ex] on the
tensor-core path, DNA and protein, with a page-locked output): bands of rows computed last
band first, each band's finished rows and mirror columns copied while the next
band is uploaded and computed, saturated tiles fixed and copied again at the
end.  Every result must be bit-identical to the unstreamed call (same kernels,
one download) and agree with the oracle like every other distance path.
"""
import numpy as np
import pytest

from oracle import oracle
from rapidnj_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def locked(n, fill=7.0):
    """An n x n float32 matrix in page-locked host memory (the streamed path's
    precondition), prefilled so that a cell the call never writes shows."""
    return torch.full((n, n), fill, dtype=torch.float32).pin_memory().numpy()


def streamed_vs_plain(ctx, seqs, model, band_tiles, type_="dna", **kw):
    n = seqs.shape[0]
    got, mx = ctx.distance_matrix_host(seqs, model, type_=type_, out=locked(n),
                                       band_tiles=band_tiles, **kw)
    ref, rmx = ctx.distance_matrix_host(seqs, model, type_=type_, band_tiles=-1, **kw)
    assert np.array_equal(got.view(np.int32), ref.view(np.int32)), \
        f"cells differ: {np.argwhere(got.view(np.int32) != ref.view(np.int32))[:5]}"
    assert mx == rmx
    return got, mx


@pytest.mark.parametrize("n,L,band_tiles", [
    (257, 300, 1),      # 3 tile rows, last tile row of one sequence
    (700, 1000, 1),     # 6 bands of one tile row
    (700, 1000, 2),     # bands of two, the last one short
    (1000, 513, 3),     # L not a multiple of 256
    (1300, 2000, 4),
    (1536, 777, 5),     # n a multiple of 128
    (2100, 4096, 0),    # the library's band height
])
@pytest.mark.parametrize("model", ["kim", "jc"])
def test_streamed_equals_unstreamed(ctx, n, L, band_tiles, model):
    seqs = synth.tree_dna(n, L, seed=n + L, mean_branch=0.05)
    streamed_vs_plain(ctx, seqs, model, band_tiles)


def test_streamed_against_oracle(ctx):
    seqs = synth.tree_dna(600, 700, seed=5, mean_branch=0.08)
    got, mx = streamed_vs_plain(ctx, seqs, "kim", 1)
    c = oracle.counts(seqs, oracle.DNA)
    ref, rmx = oracle.matrix(c, seqs.shape[1], oracle.DNA, oracle.KIMURA)
    d = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert d.max() <= 1 and (d == 1).sum() <= 2
    assert mx == np.float32(rmx)


def test_streamed_saturation_few_tiles(ctx):
    # Related sequences plus one unrelated one: K2P saturates (-1) for many
    # pairs of the unrelated sequence, so the 11 tiles of its tile row and
    # column (of 66) are fixed and copied again one by one.
    seqs = synth.tree_dna(1300, 800, seed=11, mean_branch=0.03)
    seqs[650] = synth.iid_dna(1, 800, gap=0.0, seed=12)[0]
    got, mx = streamed_vs_plain(ctx, seqs, "kim", 1)
    assert mx > 0
    # every saturated cell became 2 x max in the host copy (no -1 left)
    assert not (got == -1.0).any()
    assert (got == np.float32(2.0) * np.float32(mx)).any()


def test_streamed_saturation_everywhere(ctx):
    # Unrelated random sequences: the first band (the last rows) already shows
    # saturation in most tiles, so the call defers its download until after
    # the fix-up.
    seqs = synth.iid_dna(800, 600, gap=0.0, seed=3)
    got, mx = streamed_vs_plain(ctx, seqs, "kim", 2)
    assert not (got == -1.0).any()


def test_streamed_saturation_after_first_band(ctx):
    # Saturation only in the first rows (processed last): the bands stream out,
    # and since most tiles end up flagged the whole matrix is copied again
    # after the fix-up.
    seqs = synth.tree_dna(1300, 700, seed=8, mean_branch=0.03)
    seqs[:640] = synth.iid_dna(640, 700, gap=0.0, seed=9)
    got, mx = streamed_vs_plain(ctx, seqs, "kim", 1)
    assert not (got == -1.0).any()
    assert (got == np.float32(2.0) * np.float32(mx)).any()


def test_pageable_output_falls_back(ctx):
    # Pageable memory cannot be written by the device directly: the call takes
    # the unstreamed path and gives the same matrix.
    seqs = synth.tree_dna(500, 400, seed=2)
    out = np.full((500, 500), 5.0, dtype=np.float32)
    got, mx = ctx.distance_matrix_host(seqs, "kim", type_="dna", out=out, band_tiles=1)
    ref, rmx = ctx.distance_matrix_host(seqs, "kim", type_="dna", out=locked(500), band_tiles=-1)
    assert np.array_equal(got, ref) and mx == rmx


def test_streamed_repeated_calls_reuse_context(ctx):
    # Two different shapes one after another on the same context (the side
    # streams, the flag words and the packed-count buffer are reused).
    a = synth.tree_dna(640, 300, seed=21)
    b = synth.tree_dna(1100, 900, seed=22)
    for seqs in (a, b, a):
        streamed_vs_plain(ctx, seqs, "kim", 2)


# Protein: the whole alignment is uploaded and its residues ranked first, then
# the same bands run on the one-hot tensor-core features.
@pytest.mark.parametrize("n,L,band_tiles", [
    (257, 300, 1),
    (700, 1000, 2),
    (1000, 513, 3),
    (1536, 640, 0),     # L % 128 == 0
])
@pytest.mark.parametrize("model", ["kim", "jc"])
def test_streamed_protein_equals_unstreamed(ctx, n, L, band_tiles, model):
    seqs = synth.tree_protein(n, L, seed=n + 3 * L, mean_branch=0.15)
    streamed_vs_plain(ctx, seqs, model, band_tiles, type_="protein")


def test_streamed_protein_against_oracle(ctx):
    seqs = synth.tree_protein(600, 700, seed=6, mean_branch=0.2)
    got, mx = streamed_vs_plain(ctx, seqs, "kim", 1, type_="protein")
    c = oracle.counts(seqs, oracle.PROTEIN)
    ref, rmx = oracle.matrix(c, seqs.shape[1], oracle.PROTEIN, oracle.KIMURA)
    d = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
    assert d.max() <= 1 and (d == 1).sum() <= 2
    assert mx == np.float32(rmx)


@pytest.mark.parametrize("fastdist,compat_wrap", [(False, False), (True, True)])
def test_streamed_protein_flags(ctx, fastdist, compat_wrap):
    # The naive estimator's rules and the wrapping valid-site arithmetic of the
    # fast protein estimator (L % 128 == 0) go through the same bands.
    seqs = synth.tree_protein(900, 512, seed=17, mean_branch=0.3)
    streamed_vs_plain(ctx, seqs, "kim", 2, type_="protein", fastdist=fastdist,
                      compat_wrap=compat_wrap)


def test_streamed_protein_saturated(ctx):
    # Unrelated random proteins: distances past the table's end are fixed to
    # 2 x max after the bands.
    seqs = synth.iid_protein(800, 400, gap=0.05, seed=4)
    got, mx = streamed_vs_plain(ctx, seqs, "kim", 2, type_="protein")
    assert not (got == -1.0).any()


def test_streamed_protein_many_residues_falls_back(ctx):
    # 32 distinct residue bytes exceed the tensor-core features: the call takes
    # the bit-plane path unstreamed and gives the same matrix.
    alphabet = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWYOUacdefghikl", dtype=np.uint8)
    rng = np.random.default_rng(5)
    seqs = alphabet[rng.integers(0, alphabet.size, (500, 300))]
    streamed_vs_plain(ctx, seqs, "kim", 1, type_="protein")
