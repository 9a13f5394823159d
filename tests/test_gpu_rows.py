"""rnj_distance_rows: distance matrices delivered in bands of full rows, with
device buffers for two bands only (matrices larger than device memory).

rapidNJ's disk-matrix drivers compute every row in full and post-process the
rows once the maximum is known (KimuraDistance.cpp:308-354, 366-395;
JCdistance.cpp:160-195, 201-230).  The delivered rows, post-processed the same
way (-1 -> 2 * max), must equal the in-memory matrix of the library bit for bit
and the oracle's matrix within the parity rule (<= 1 ulp, rare), for every
counting kernel: the tensor cores (DNA, protein), the bit planes (-f DNA with
its asymmetric counts, protein alphabets beyond the tensor-core limit), with
saturated pairs, and band heights from one tile to more than the matrix.
"""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def ulp_diff(a, b):
    a = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def rows_matrix(ctx, aln, model, band_rows):
    n = aln.n
    out = np.full((n, n), np.nan, np.float32)
    seen = []

    def on_rows(row0, rows):
        seen.append((row0, rows.shape[0]))
        out[row0:row0 + rows.shape[0]] = rows

    mx, sat = ctx.distance_rows(aln, model, on_rows, band_rows)
    # in row order, every row once
    assert [r for r, _ in seen] == sorted(r for r, _ in seen)
    assert sum(k for _, k in seen) == n and not np.isnan(out).any()
    assert (np.diagonal(out) == 0).all()
    assert sat == bool((out == -1).any())
    return np.where(out == -1, np.float32(2) * np.float32(mx), out), mx


def crafted(kind):
    from rapidnj_b200 import synth
    rng = np.random.default_rng(5)
    if kind == "dna":
        return synth.tree_dna(300, 700, seed=1, mean_branch=0.1), oracle.DNA, {}
    if kind == "dna-saturated":
        return np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (260, 40))], oracle.DNA, {}
    if kind == "protein":
        return synth.tree_protein(270, 500, seed=2, mean_branch=0.3), oracle.PROTEIN, {}
    if kind == "dna-naive":
        s = synth.tree_dna(250, 600, seed=3, mean_branch=0.1)
        s[rng.random(s.shape) < 0.1] = ord("a")
        s[rng.random(s.shape) < 0.02] = ord("U")
        return s, oracle.DNA, {"fastdist": False, "full_rows": True}
    if kind == "protein-80":
        a = np.frombuffer(bytes(range(40, 120)), np.uint8)
        s = a[rng.integers(0, a.size, (200, 300))]
        s[rng.random(s.shape) < 0.05] = ord("-")
        return s, oracle.PROTEIN, {}
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["dna", "dna-saturated", "protein", "dna-naive", "protein-80"])
@pytest.mark.parametrize("model", ["kim", "jc"])
@pytest.mark.parametrize("band_rows", [128, 256, 0, 4096])
def test_row_bands_equal_in_memory_matrix_and_oracle(ctx, kind, model, band_rows):
    seqs, typ, opts = crafted(kind)
    aln = ctx.alignment(seqs, typ, **opts)
    got, mx = rows_matrix(ctx, aln, model, band_rows)
    mat = ctx.distance(aln, model)
    want, wmx = mat.to_numpy(), mat.max
    mat.close()
    aln.close()
    assert mx == wmx
    assert np.array_equal(got.view(np.int32), want.view(np.int32))
    naive = not opts.get("fastdist", True)
    c = oracle.counts(seqs, typ, naive=naive, full=naive, threads=8)
    ref, rmx = oracle.matrix(c, seqs.shape[1], typ, oracle.JC if model == "jc" else oracle.KIMURA,
                             naive=naive, full=naive)
    d = ulp_diff(got, ref)
    assert d.max() <= 1 and (d == 1).sum() <= 2


def test_row_bands_of_the_large_workload_shape(ctx):
    """Several bands of a 3,000 x 2,000 DNA alignment (bands of 512 rows of 3,000
    floats), against the in-memory matrix."""
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(3000, 2000, seed=9)
    aln = ctx.alignment(torch.from_numpy(seqs).cuda(), oracle.DNA)
    got, mx = rows_matrix(ctx, aln, "kim", 512)
    out = torch.empty((3000, 3000), dtype=torch.float32, device="cuda")
    wmx = ctx.distance_into(aln, "kim", out, want_max=True)
    aln.close()
    assert mx == wmx and np.array_equal(got, out.cpu().numpy())


def test_row_bands_stop_when_the_callback_fails(ctx):
    from rapidnj_b200 import synth
    from rapidnj_b200._native import RnjError
    seqs = synth.tree_dna(400, 300, seed=4)
    aln = ctx.alignment(seqs, oracle.DNA)

    def boom(row0, rows):
        if row0 > 0:
            raise RuntimeError("stop")

    with pytest.raises(RuntimeError):
        ctx.distance_rows(aln, "kim", boom, 128)
    # the context is usable afterwards
    got, _ = rows_matrix(ctx, aln, "kim", 128)
    mat = ctx.distance(aln, "kim")
    assert np.array_equal(got, mat.to_numpy())
    mat.close()
    aln.close()
    with pytest.raises(RnjError):
        ctx.distance_rows(aln, "kim", lambda r0, r: None, -1)
