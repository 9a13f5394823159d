"""Packing reads device rows of any alignment: base pointers at every byte
offset from a 16-byte boundary and row strides that are not multiples of 16,
through the DNA and protein feature packs, the residue-presence scan and the
batched pack.  The bytes between rows are residues, so a read outside a row
would change the counts; every count must equal the oracle's bit for bit."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def device_view(seqs, offset, pad, fill):
    """seqs as an (n, L) CUDA view whose first byte is `offset` bytes past a
    256-byte boundary and whose stride is L + pad, the bytes around the rows
    set to `fill`."""
    n, L = seqs.shape
    ld = L + pad
    buf = torch.full((offset + n * ld + 64,), fill, dtype=torch.uint8, device="cuda")
    assert buf.data_ptr() % 256 == 0
    rows = buf[offset:offset + n * ld].view(n, ld)
    rows[:, :L] = torch.from_numpy(seqs).cuda()
    view = rows[:, :L]
    assert view.data_ptr() % 16 == offset % 16 and view.stride(0) == ld
    return view


def counts_of(ctx, view, typ):
    aln = ctx.alignment(view, typ)
    n = view.shape[0]
    out = torch.zeros(n * n * 3, dtype=torch.int32, device="cuda")
    ctx.counts_into(aln, out)
    aln.close()
    return out.cpu().numpy().view(np.uint32).reshape(n, n, 3)


CASES = [(0, 0), (1, 3), (5, 7), (8, 1), (13, 0), (15, 17), (3, 16)]


@pytest.mark.parametrize("offset,pad", CASES)
@pytest.mark.parametrize("L", [1, 17, 31, 33, 300, 1001])
def test_dna_rows_at_any_alignment(ctx, offset, pad, L):
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(70, L, seed=L + offset, mean_branch=0.15)
    view = device_view(seqs, offset, pad, ord("A"))
    assert np.array_equal(counts_of(ctx, view, oracle.DNA), oracle.counts(seqs, oracle.DNA))


@pytest.mark.parametrize("offset,pad", CASES)
@pytest.mark.parametrize("L", [1, 15, 32, 47, 513, 4100, 9000])
def test_protein_rows_at_any_alignment(ctx, offset, pad, L):
    """L past 4096 puts a row in two presence segments; a residue that occurs
    only in the last column (or only in the first) must still be ranked."""
    from rapidnj_b200 import synth
    seqs = synth.tree_protein(60, L, seed=L + 3 * offset, mean_branch=0.3)
    seqs[-1, -1] = ord("W")
    seqs[0, 0] = ord("Y")
    # 'O' only in the padding: it must not be seen (no rank, no count)
    view = device_view(seqs, offset, pad, ord("O"))
    assert np.array_equal(counts_of(ctx, view, oracle.PROTEIN),
                          oracle.counts(seqs, oracle.PROTEIN))


def test_protein_rare_residue_at_row_ends(ctx):
    """Residues that occur once, at an unaligned row start and at a row end,
    get their own rank (the presence scan's byte-by-byte ends)."""
    from rapidnj_b200 import synth
    seqs = synth.tree_protein(40, 777, seed=9, mean_branch=0.2)
    seqs[seqs == ord("M")] = ord("A")
    seqs[seqs == ord("C")] = ord("A")
    seqs[17, 0] = ord("M")
    seqs[23, 776] = ord("C")
    view = device_view(seqs, 7, 5, ord("-"))
    assert np.array_equal(counts_of(ctx, view, oracle.PROTEIN),
                          oracle.counts(seqs, oracle.PROTEIN))


def test_batched_pack_of_unaligned_rows(ctx):
    """add_many over device views at odd offsets and strides, DNA and protein
    mixed: the batched presence scan and feature pack give the oracle's
    matrices."""
    from rapidnj_b200 import api, synth
    rng = np.random.default_rng(4)
    seqs, types, views = [], [], []
    for k in range(12):
        n, L = int(rng.integers(2, 300)), int(rng.integers(1, 2500))
        prot = k % 3 == 0
        s = (synth.tree_protein(n, L, seed=k) if prot
             else synth.tree_dna(n, L, seed=k, mean_branch=0.15))
        seqs.append(s)
        types.append(1 if prot else 0)
        views.append(device_view(s, int(rng.integers(0, 16)), int(rng.integers(0, 20)),
                                 ord("O") if prot else ord("C")))
    batch = api.Batch(ctx, max_alignments=16, max_tiles=512)
    slots = batch.add_many(views, types, ["kim"] * len(views))
    batch.run()
    for s, t, slot in zip(seqs, types, slots):
        typ = oracle.PROTEIN if t else oracle.DNA
        ref, _ = oracle.matrix(oracle.counts(s, typ), s.shape[1], typ, oracle.KIMURA)
        got = batch.take(slot).to_numpy()
        d = np.abs(got.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64))
        assert d.max(initial=0) <= 1 and (d == 1).sum() <= max(2, int(1e-6 * d.size))
    batch.close()
