"""Parity of the sm_100a path (through the C ABI) with the reference.

* counts: bit-exact against the reference's goldens and the pinned oracle;
* distances: the float matrices of the reference.  The only allowed difference
  is CUDA's double log() against glibc's (both within 1 ulp in double), which can
  move a float result by one ulp in rare cells: the tests require every cell
  within 1 float ulp and at most max(2, 1e-6 * cells) cells off by that ulp.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_files, golden_type, load_golden
from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

GOLDENS = golden_files()


def ulp_diff(a, b):
    a = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    # map sign-magnitude to a monotone integer line
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def assert_matrix_parity(got, ref):
    assert got.shape == ref.shape
    d = ulp_diff(got, ref)
    assert d.max(initial=0) <= 1, f"cells beyond 1 ulp: {np.argwhere(d > 1)[:5]}"
    assert (d == 1).sum() <= max(2, int(1e-6 * d.size)), f"{(d == 1).sum()} one-ulp cells"


def gpu_counts(ctx, seqs, typ, fastdist=True, full_rows=False, popcount=False):
    aln = ctx.alignment(seqs, typ, fastdist=fastdist, full_rows=full_rows, popcount=popcount)
    n = seqs.shape[0]
    out = torch.zeros(n * n * 3, dtype=torch.int32, device="cuda")
    ctx.counts_into(aln, out)
    aln.close()
    return out.cpu().numpy().view(np.uint32).reshape(n, n, 3)


def gpu_matrix(ctx, seqs, typ, model, fastdist=True, compat_wrap=False, full_rows=False,
               popcount=False):
    aln = ctx.alignment(seqs, typ, fastdist=fastdist, compat_wrap=compat_wrap, full_rows=full_rows,
                        popcount=popcount)
    mat = ctx.distance(aln, model)
    out, mx = mat.to_numpy(), mat.max
    mat.close()
    aln.close()
    return out, mx


# ----------------------------------------------------------------- goldens

@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
@pytest.mark.parametrize("popcount", [False, True], ids=["default", "popcount"])
def test_counts_match_reference(ctx, path, popcount):
    g = load_golden(path)
    seqs, typ = g["chars"], golden_type(g)
    L = seqs.shape[1]
    fast = gpu_counts(ctx, seqs, typ, popcount=popcount)
    if typ == oracle.PROTEIN and L % 128 == 0:
        # the reference fast estimator's valid count is wrong here; ours is the
        # naive estimator's, which is correct
        assert np.array_equal(fast, g["counts_naive"])
    else:
        assert np.array_equal(fast, g["counts_fast"])
    assert np.array_equal(gpu_counts(ctx, seqs, typ, fastdist=False), g["counts_naive"])
    assert np.array_equal(gpu_counts(ctx, seqs, typ, fastdist=False, full_rows=True),
                          g["counts_naive_full"])


@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
@pytest.mark.parametrize("model", ["jc", "kim"])
@pytest.mark.parametrize("popcount", [False, True], ids=["default", "popcount"])
def test_matrices_match_reference(ctx, path, model, popcount):
    g = load_golden(path)
    seqs, typ = g["chars"], golden_type(g)
    L = seqs.shape[1]
    got, _ = gpu_matrix(ctx, seqs, typ, model, popcount=popcount)
    if typ == oracle.PROTEIN and L % 128 == 0:
        assert_matrix_parity(got, g[f"{model}_naive"])
        wrapped, _ = gpu_matrix(ctx, seqs, typ, model, compat_wrap=True)
        assert_matrix_parity(wrapped, g[f"{model}_fast"])
    else:
        assert_matrix_parity(got, g[f"{model}_fast"])
    naive, _ = gpu_matrix(ctx, seqs, typ, model, fastdist=False)
    assert_matrix_parity(naive, g[f"{model}_naive"])


@pytest.mark.parametrize("path", GOLDENS, ids=lambda p: p.split("/")[-1])
def test_disk_row_mode_matches_reference(ctx, path):
    g = load_golden(path)
    seqs, typ = g["chars"], golden_type(g)
    got, _ = gpu_matrix(ctx, seqs, typ, "kim", fastdist=False, full_rows=True)
    assert_matrix_parity(got, g["kim_naive_disk"])


# --------------------------------------------------- random shapes vs oracle

SHAPES = [(1, 10), (2, 1), (3, 31), (5, 32), (17, 33), (127, 255), (128, 256), (129, 257),
          (200, 1000), (300, 4096), (257, 65)]


@pytest.mark.parametrize("n,L", SHAPES)
@pytest.mark.parametrize("kind", ["dna", "dna-popcount", "protein"])
def test_random_alignments_vs_oracle(ctx, n, L, kind):
    from rapidnj_b200 import synth
    seed = n * 1000 + L
    seqs = synth.tree_dna(n, L, seed=seed, mean_branch=0.1) if kind != "protein" else \
        synth.tree_protein(n, L, seed=seed, mean_branch=0.3)
    typ = oracle.DNA if kind != "protein" else oracle.PROTEIN
    pc = kind == "dna-popcount"
    c = oracle.counts(seqs, typ)
    assert np.array_equal(gpu_counts(ctx, seqs, typ, popcount=pc), c)
    for model, mo in (("jc", oracle.JC), ("kim", oracle.KIMURA)):
        ref, rmax = oracle.matrix(c, L, typ, mo)
        got, gmax = gpu_matrix(ctx, seqs, typ, model, popcount=pc)
        assert_matrix_parity(got, ref)
        assert abs(gmax - rmax) <= 1e-6 * max(1.0, rmax)


@pytest.mark.parametrize("alphabet", [b"ACGT", b"ARNDCQEGHILKMFPSTWYV", bytes(range(40, 120))])
def test_protein_alphabet_sizes(ctx, alphabet):
    rng = np.random.default_rng(len(alphabet))
    a = np.frombuffer(alphabet, np.uint8)
    seqs = a[rng.integers(0, a.size, (150, 700))]
    seqs[rng.random(seqs.shape) < 0.05] = ord("-")
    c = oracle.counts(seqs, oracle.PROTEIN)
    assert np.array_equal(gpu_counts(ctx, seqs, oracle.PROTEIN), c)
    ref, _ = oracle.matrix(c, 700, oracle.PROTEIN, oracle.KIMURA)
    got, _ = gpu_matrix(ctx, seqs, oracle.PROTEIN, "kim")
    assert_matrix_parity(got, ref)


@pytest.mark.parametrize("kind", ["dna", "protein"])
def test_long_alignment_split_path(ctx, kind):
    """L > 65504 takes the split-K count path (atomic partial counts + transform)."""
    from rapidnj_b200 import synth
    n, L = 40, 70001
    seqs = synth.tree_dna(n, L, seed=3, mean_branch=0.2) if kind == "dna" else \
        synth.tree_protein(n, L, seed=3, mean_branch=0.4)
    typ = oracle.DNA if kind == "dna" else oracle.PROTEIN
    c = oracle.counts(seqs, typ)
    assert np.array_equal(gpu_counts(ctx, seqs, typ), c)
    ref, _ = oracle.matrix(c, L, typ, oracle.KIMURA)
    got, _ = gpu_matrix(ctx, seqs, typ, "kim")
    assert_matrix_parity(got, ref)


def test_saturation_fixup(ctx):
    """Unrelated sequences saturate (-1 -> 2 * max) exactly as the reference."""
    rng = np.random.default_rng(9)
    seqs = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (300, 40))]
    c = oracle.counts(seqs, oracle.DNA)
    for model, mo in (("jc", oracle.JC), ("kim", oracle.KIMURA)):
        ref, mx = oracle.matrix(c, 40, oracle.DNA, mo)
        got, gmx = gpu_matrix(ctx, seqs, oracle.DNA, model)
        assert (ref == 2 * mx).sum() > 0
        assert_matrix_parity(got, ref)


@pytest.mark.parametrize("model,mo", [("kim", oracle.KIMURA), ("jc", oracle.JC)])
def test_saturation_fixup_of_a_large_triangle(ctx, model, mo):
    """A triangle of 4,465 tiles, about half its pairs saturated: no -1 is
    left, saturated cells hold 2 x the global maximum, the others the
    reference's value (cells among 240 random sequences, against the oracle's
    counts)."""
    n, L = 12000, 48
    rng = np.random.default_rng(31)
    seqs = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (n, L))]
    aln = ctx.alignment(torch.from_numpy(seqs).cuda(), oracle.DNA)
    out = torch.empty((n, n), dtype=torch.float32, device="cuda")
    mx = ctx.distance_into(aln, model, out, want_max=True)
    aln.close()
    rows = np.sort(rng.choice(n, 240, replace=False))
    got = out[torch.from_numpy(rows).cuda()][:, torch.from_numpy(rows).cuda()].cpu().numpy()
    assert not bool((out == -1.0).any())
    del out
    ref, rmx = oracle.matrix(oracle.counts(seqs[rows], oracle.DNA), L, oracle.DNA, mo)
    off = ~np.eye(len(rows), dtype=bool)
    sat = (ref == np.float32(2.0) * np.float32(rmx)) & off
    assert sat.sum() > 1000
    assert (got[sat] == np.float32(2.0) * np.float32(mx)).all()
    d = ulp_diff(got[~sat], ref[~sat])
    assert d.max() <= 1 and (d == 1).sum() <= 2


def test_all_saturated_gives_zero_matrix(ctx):
    seqs = np.array([list(b"AAAA"), list(b"TTTT"), list(b"CCCC")], np.uint8)
    got, mx = gpu_matrix(ctx, seqs, oracle.DNA, "kim")
    assert mx == 0.0 and not got.any()


# ----------------------------------------------------------- input paths

def reference_bitstrings(seqs):
    """The reference loader's DNA layout (dataloaderFasta.hpp:147-182, 219-240):
    bitStringsCount = L/64 + 6 vectors of 4 uint32, 16 sites per word."""
    n, L = seqs.shape
    count = L // 64 + 6
    code = {ord("A"): 0, ord("a"): 0, ord("G"): 1, ord("g"): 1, ord("T"): 2, ord("t"): 2,
            ord("C"): 3, ord("c"): 3}
    bs, gf = [], []
    for i in range(n):
        b = np.zeros(count * 4, np.uint32)
        g = np.zeros(count * 4, np.uint32)
        for k in range(L):
            c = int(seqs[i, k])
            if c in code:
                b[k // 16] |= np.uint32(code[c] << (2 * (k % 16)))
                g[k // 16] |= np.uint32(1 << (2 * (k % 16)))
        bs.append(b)
        gf.append(g)
    return bs, gf


def test_input_paths_agree(ctx):
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(150, 777, seed=11, mean_branch=0.1)
    ref, _ = gpu_matrix(ctx, seqs, oracle.DNA, "kim")
    # row pointers
    aln = ctx.alignment_from_rows([r.tobytes() for r in seqs], oracle.DNA)
    m = ctx.distance(aln, "kim")
    assert np.array_equal(m.to_numpy(), ref)
    # device tensor with a padded stride
    t = torch.zeros((150, 800), dtype=torch.uint8, device="cuda")
    t[:, :777] = torch.from_numpy(seqs).cuda()
    aln = ctx.alignment(t[:, :777], oracle.DNA)
    assert np.array_equal(ctx.distance(aln, "kim").to_numpy(), ref)
    # the reference loader's bit strings
    bs, gf = reference_bitstrings(seqs)
    aln = ctx.alignment_from_bitstrings(bs, gf, 777, oracle.DNA)
    assert np.array_equal(ctx.distance(aln, "kim").to_numpy(), ref)
    # ... on the popcount kernel, and the JC model on both kernels
    from rapidnj_b200.api import RNJ_FASTDIST, RNJ_POPCOUNT
    aln_p = ctx.alignment_from_bitstrings(bs, gf, 777, oracle.DNA, RNJ_FASTDIST | RNJ_POPCOUNT)
    assert np.array_equal(ctx.distance(aln_p, "kim").to_numpy(), ref)
    ref_jc, _ = gpu_matrix(ctx, seqs, oracle.DNA, "jc")
    assert np.array_equal(ctx.distance(aln, "jc").to_numpy(), ref_jc)
    assert np.array_equal(ctx.distance(aln_p, "jc").to_numpy(), ref_jc)
    # one-call host path, into pageable and into page-locked host memory
    out, mx = ctx.distance_matrix_host(seqs, "kim")
    assert np.array_equal(out, ref)
    locked = torch.full((150, 150), 3.0, dtype=torch.float32).pin_memory().numpy()
    _, mx_locked = ctx.distance_matrix_host(seqs, "kim", out=locked)
    assert np.array_equal(locked, ref) and mx_locked == mx
    # caller-owned device buffer with a stride
    buf = torch.full((150, 160), 7.0, dtype=torch.float32, device="cuda")
    mx2 = ctx.distance_into(ctx.alignment(seqs, oracle.DNA), "kim", buf, want_max=True)
    assert np.array_equal(buf[:, :150].cpu().numpy(), ref) and mx2 == mx
    assert (buf[:, 150:] == 7.0).all()


def test_reference_interface(ctx, tmp_path):
    """JCdistance / KimuraDistance as rapidNJ's driver calls them (main.cpp:259-270)."""
    from rapidnj_b200 import Dataloader, JCdistance, KimuraDistance
    g = load_golden(f"{oracle.HERE}/../tests/golden/fixture_LGT_70.npz")
    f = tmp_path / "LGT_70.fa"
    f.write_bytes(bytes(g["fa_text"]))
    dl = Dataloader()
    dl.readData(str(f), True, False)
    alg = JCdistance(False, True, dl, None, ctx=ctx)
    alg.computeDistanceMatrix(4)
    assert_matrix_parity(alg.getDistanceMatrix(), g["jc_fast"])
    alg = KimuraDistance(False, True, dl, None, ctx=ctx)
    alg.computeDistances(4)
    assert_matrix_parity(alg.getDistanceMatrix(), g["kim_fast"])

    class Rows:
        def __init__(self, n):
            self.rows = np.zeros((n, n), np.float32)

        def writeArray(self, row, i, n):
            self.rows[i] = row[:n]

    dm = Rows(dl.getSequenceCount())
    KimuraDistance(False, True, dl, dm, ctx=ctx).computeDistances(2)
    assert_matrix_parity(dm.rows, g["kim_fast_disk"])


def test_repeatable(ctx):
    from rapidnj_b200 import synth
    seqs = synth.tree_protein(400, 1500, seed=4)
    a, _ = gpu_matrix(ctx, seqs, oracle.PROTEIN, "kim")
    b, _ = gpu_matrix(ctx, seqs, oracle.PROTEIN, "kim")
    assert np.array_equal(a, b)


# ------------------------------------------------------------ full size

def test_full_size_k2p_properties(ctx):
    """10,000 x 10,000 tree-evolved DNA: symmetric, zero diagonal, no sentinel
    left, max consistent, and 3,000 sampled pairs equal to the oracle."""
    from rapidnj_b200 import synth
    n, L = 10000, 10000
    seqs = synth.tree_dna(n, L, seed=0)
    t = torch.from_numpy(seqs).cuda()
    aln = ctx.alignment(t, oracle.DNA)
    out = torch.empty((n, n), dtype=torch.float32, device="cuda")
    mx = ctx.distance_into(aln, "kim", out, want_max=True)
    assert torch.equal(out, out.T)
    assert (out.diagonal() == 0).all()
    assert not (out == -1).any()
    assert float(out.max()) == max(mx, 2 * mx if (out == 2 * mx).any() else mx)
    rng = np.random.default_rng(1)
    ii = rng.integers(0, n, 3000)
    jj = rng.integers(0, n, 3000)
    lib = oracle.lib()
    lib.orc_pair_counts.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.POINTER(ctypes.c_uint64)]
    lib.orc_distance.argtypes = [ctypes.POINTER(ctypes.c_uint32), ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.orc_distance.restype = ctypes.c_float
    got = out[torch.from_numpy(ii).cuda(), torch.from_numpy(jj).cuda()].cpu().numpy()
    exp = np.empty(3000, np.float32)
    c64 = (ctypes.c_uint64 * 3)()
    for k, (i, j) in enumerate(zip(ii, jj)):
        if i == j:
            exp[k] = 0.0
            continue
        lib.orc_pair_counts(seqs[i].tobytes(), seqs[j].tobytes(), L, 0, 0, c64)
        c32 = (ctypes.c_uint32 * 3)(*[int(x) for x in c64])
        d = lib.orc_distance(c32, L, 0, 1, 0, 0)
        exp[k] = 2 * mx if d == -1 else d
    assert ulp_diff(got, exp).max() <= 1


def test_full_size_k2p_matrix_vs_reference(ctx, tmp_path):
    """The whole 10,000 x 10,000 Kimura-2P matrix of the benchmark workload, cell
    for cell against the float matrix of the reference's own driver
    (KimuraDistance::computeDistances, KimuraDistance.cpp:300-395, compiled from
    the reference sources into oracle/_ref/ref_harness, all host threads)."""
    import os
    from rapidnj_b200 import synth
    if not oracle.ref_available():
        pytest.skip("reference harness not built")
    n, L = 10000, 10000
    seqs = synth.tree_dna(n, L, seed=0)
    path = str(tmp_path / "bench.fa")
    synth.write_fasta(path, seqs)
    ref, info = oracle.ref_matrix(path, "kim", "fa", "d", True, threads=os.cpu_count() or 1)
    assert ref.shape == (n, n) and info["n"] == n and info["L"] == L
    aln = ctx.alignment(torch.from_numpy(seqs).cuda(), oracle.DNA)
    out = torch.empty((n, n), dtype=torch.float32, device="cuda")
    ctx.distance_into(aln, "kim", out)
    aln.close()
    got = out.cpu().numpy()
    del out
    worst, ones = 0, 0
    for r0 in range(0, n, 1000):  # row bands: the ulp arithmetic needs int64 copies
        d = ulp_diff(got[r0:r0 + 1000], ref[r0:r0 + 1000])
        worst = max(worst, int(d.max()))
        ones += int((d == 1).sum())
    assert worst <= 1, f"a cell differs by {worst} ulp"
    assert ones <= max(2, int(1e-6 * n * n)), f"{ones} one-ulp cells"


def test_tensor_core_exact_at_column_cap(ctx):
    """The tensor-core path takes DNA up to 2^21 - 1 columns, where the f32 sums
    of the FP4 products reach 2L ~ 2^22 in magnitude: nearly identical sequences
    without gaps (and exact copies, whose T sum is exactly 2L) must still give the
    oracle's integer counts and distances."""
    import os
    from rapidnj_b200 import synth
    n, L = 130, (1 << 21) - 1
    seqs = synth.tree_dna(n, L, seed=17, mean_branch=0.0004, gap=0.0)
    seqs[1] = seqs[0]                      # identical: V = R = L, T = 2L
    seqs[2, : L // 2] = seqs[3, : L // 2]  # half copied
    seqs[4, 1::2] = ord("-")               # every other site a gap
    c = oracle.counts(seqs, oracle.DNA, threads=os.cpu_count() or 1)
    assert c[0, 1, 2] == L and c[0, 1, 0] == 0 and c[0, 1, 1] == 0
    got = gpu_counts(ctx, seqs, oracle.DNA)
    assert np.array_equal(got, c)
    ref, _ = oracle.matrix(c, L, oracle.DNA, oracle.KIMURA)
    m, _ = gpu_matrix(ctx, seqs, oracle.DNA, "kim")
    assert_matrix_parity(m, ref)


# ------------------------------------------------- tensor-core DNA kernel

TC_SHAPES = [(2, 1), (3, 31), (17, 127), (128, 128), (129, 129), (200, 1000), (257, 4097),
             (300, 300), (1, 5)]


@pytest.mark.parametrize("n,L", TC_SHAPES)
def test_tensor_core_counts_vs_oracle(ctx, n, L):
    """DNA on the fast path runs on the tensor cores by default."""
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(n, L, seed=n + 7 * L, mean_branch=0.15)
    assert np.array_equal(gpu_counts(ctx, seqs, oracle.DNA), oracle.counts(seqs, oracle.DNA))


def test_tensor_core_full_rows_counts(ctx):
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(150, 500, seed=5, mean_branch=0.2)
    got = gpu_counts(ctx, seqs, oracle.DNA, full_rows=True)
    assert np.array_equal(got, oracle.counts(seqs, oracle.DNA, full=True))


def test_tensor_core_matches_popcount_kernel(ctx):
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(1000, 3000, seed=21)
    for model in ("jc", "kim"):
        a, am = gpu_matrix(ctx, seqs, oracle.DNA, model, popcount=True)
        b, bm = gpu_matrix(ctx, seqs, oracle.DNA, model)
        assert np.array_equal(a, b) and am == bm
