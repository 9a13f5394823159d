"""rnj_nj_init on the device: rapidNJ's set-up over a distance matrix (separation
sums in the reference's order, separations, running maximum, redundant rows,
sorted rows).  Against the reference's own results (tests/golden/nj_*.npz) with
equal-distance runs compared as sets, and against the oracle exactly."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle
from njcheck import bits, compare, device_rows, golden
from rapidnj_b200 import synth

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "nj_*.npz")))


def run(ctx, m, cap, ld_pad=0):
    n = m.shape[0]
    buf = torch.full((n, n + ld_pad), 3.0, dtype=torch.float32, device="cuda")
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(m, dtype=np.float32)).cuda()
    res = ctx.nj_init(buf[:, :n], cap=cap)
    res["sums"] = res["separation_sums"]
    res["rows"] = device_rows(res)
    return res


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[3:-4] for p in GOLDEN])
@pytest.mark.parametrize("cap", [0, 5])
def test_matches_reference_and_oracle(ctx, path, cap):
    z = np.load(path)
    got = run(ctx, z["matrix"], cap)
    compare(got, golden(z, cap), cap, exact_ties=False)
    want = oracle.nj_init(z["matrix"], cap)
    compare(got, want, cap, exact_ties=True)
    assert np.array_equal(got["possible_redundant"], want["possible_redundant"])


@pytest.mark.parametrize("n,L,cap,pad", [(700, 500, 0, 3), (1300, 300, 64, 0), (2049, 200, 0, 1)])
def test_tree_with_duplicates_against_oracle(ctx, n, L, cap, pad):
    s = synth.tree_dna(n, L, seed=n, mean_branch=0.03)
    rng = np.random.default_rng(n)
    for _ in range(n // 20):
        a, b = rng.integers(0, n, 2)
        s[a] = s[b]
    m, _ = oracle.distance_matrix(s, oracle.KIMURA, oracle.DNA)
    got = run(ctx, m, cap, pad)
    want = oracle.nj_init(m, cap)
    compare(got, want, cap, exact_ties=True)
    assert (want["redundant_count"] > 1).any()


def points_matrix(n, seed, dup=0.02, device="cuda"):
    """|x_i - x_j| over float32 points with some repeated (redundant rows) and
    many equal distances (points on a grid of 1/1024 in [0, 1024])."""
    rng = np.random.default_rng(seed)
    x = np.round(rng.random(n) * 1048576.0) / 1024.0
    k = int(n * dup)
    x[rng.integers(0, n, k)] = x[rng.integers(0, n, k)]
    t = torch.from_numpy(x.astype(np.float32)).to(device)
    return (t[:, None] - t[None, :]).abs(), x


def test_long_rows_against_oracle(ctx):
    # rows of more than 8192 entries: sorted through the global scratch row
    m, _ = points_matrix(8600, 1)
    mh = m.cpu().numpy()
    got = run(ctx, mh, 0)
    want = oracle.nj_init(mh, 0)
    assert want["row_lengths"].max() > 8192
    compare(got, want, 0, exact_ties=True)


@pytest.mark.parametrize("cap", [0, 3000])
def test_very_long_rows_properties(ctx, cap):
    # n = 17,000: rows up to 32,768 keys (two global merge strides).  Checked by
    # size-independent properties: sums equal the column-order float sums, every
    # kept row lists exactly the kept rows below it, by distance then id, with the
    # stored distances.
    n = 17000
    m, _ = points_matrix(n, 2)
    res = ctx.nj_init(m, cap=cap)
    assert (res["index_to_id"] != -1).sum() > 16385
    mh = m.cpu().numpy()
    sums = np.cumsum(mh, axis=1, dtype=np.float32)[:, -1]
    assert np.array_equal(bits(res["separation_sums"]), bits(sums))
    keep = torch.from_numpy(res["index_to_id"] != -1).cuda()
    kept_idx = torch.nonzero(keep).flatten().to(torch.int32)
    rank = torch.cumsum(keep.to(torch.int64), 0) - keep.to(torch.int64)
    full_len = torch.where(keep, rank, torch.zeros_like(rank))
    lens = torch.from_numpy(res["row_lengths"]).cuda().to(torch.int64)
    assert torch.equal(lens, full_len if cap == 0 else torch.clamp(full_len, max=cap))
    ids = res["sorted"][..., 0]
    d = res["sorted_distances"]
    W = ids.shape[1]
    pos = torch.arange(W, device="cuda")
    valid = pos[None, :] < lens[:, None]
    # stored distances
    g = torch.gather(m, 1, torch.where(valid, ids, torch.zeros_like(ids)).long())
    assert torch.equal(torch.where(valid, g, 0.0).view(torch.int32),
                       torch.where(valid, d, 0.0).view(torch.int32))
    # ascending by (distance, id)
    v2 = valid[:, 1:]
    dd, di = d[:, 1:] - d[:, :-1], ids[:, 1:] - ids[:, :-1]
    assert bool(((dd > 0) | ((dd == 0) & (di > 0)) | ~v2).all())
    if cap == 0:
        # the ids of row i are the kept rows below i
        big = torch.iinfo(torch.int32).max
        s, _ = torch.sort(torch.where(valid, ids, big), dim=1)
        ref = torch.where(valid, kept_idx[torch.clamp(pos, max=len(kept_idx) - 1)][None, :], big)
        assert torch.equal(s, ref)
    else:
        # the first cap of the full order
        full = ctx.nj_init(m, cap=0)
        assert torch.equal(torch.where(valid, ids, 0), torch.where(valid, full["sorted"][:, :W, 0], 0))


def test_nan_rows_are_not_redundant(ctx):
    # rows 5 and 20 equal but for a NaN in the same column: NaN != NaN, so neither
    # is redundant (the sums are NaN; their NaN bits are the device's, compared
    # by value here)
    m, _ = points_matrix(300, 5, dup=0.0)
    m[20] = m[5]
    m[:, 20] = m[:, 5]
    m[20, 20] = m[5, 5] = 0.0
    m[5, 9] = m[9, 5] = m[20, 9] = m[9, 20] = float("nan")
    mh = m.cpu().numpy()
    got = run(ctx, mh, 0)
    want = oracle.nj_init(mh, 0)
    assert want["index_to_id"][5] == 5 and want["index_to_id"][20] == 20
    for k in ("index_to_id", "redundant_to_master", "redundant_count", "row_lengths"):
        assert np.array_equal(got[k], want[k]), k
    assert np.array_equal(got["separation_sums"], want["sums"], equal_nan=True)


def test_non_zero_diagonal_is_rejected(ctx):
    from rapidnj_b200._native import RnjError
    m, _ = points_matrix(100, 6)
    m[7, 7] = 1.0
    with pytest.raises(RnjError, match="diagonal"):
        ctx.nj_init(m)


def test_after_distance_call(ctx):
    # the matrix the library just produced, still on the device
    s = synth.tree_dna(900, 1000, seed=9, mean_branch=0.04)
    s[10] = s[500]
    aln = ctx.alignment(torch.from_numpy(s).cuda(), 0)
    out = torch.empty((900, 900), dtype=torch.float32, device="cuda")
    ctx.distance_into(aln, "kim", out)
    aln.close()
    got = ctx.nj_init(out)
    want = oracle.nj_init(out.cpu().numpy(), 0)
    got["sums"] = got["separation_sums"]
    got["rows"] = device_rows(got)
    compare(got, want, 0, exact_ties=True)
    assert got["redundant_to_master"][10] == 500
