"""rnj_distance_f64: the matrix in double precision (each pair's value is the
reference's double before its float cast, JCdistance.cpp:171-183 and
KimuraDistance.cpp:322-349, then the post-process in double).  Checked against
the oracle's double matrix (orc_matrix_d, whose float rounding is the pinned
float matrix) within 1e-12 relative (CUDA's and glibc's double log differ by at
most an ulp; table values, 10.0, 0 and the saturation cap agree exactly), and
its float rounding against the float matrix of rnj_distance (at most one ulp in
at most max(2, 1e-6 of the cells), the rule of the float parity tests)."""
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


def case(kind):
    from rapidnj_b200 import synth
    rng = np.random.default_rng(7)
    if kind == "dna":
        return synth.tree_dna(300, 900, seed=1, mean_branch=0.1), oracle.DNA, {}
    if kind == "dna-saturated":
        return np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (200, 60))], oracle.DNA, {}
    if kind == "protein":
        return synth.tree_protein(260, 500, seed=2, mean_branch=0.3), oracle.PROTEIN, {}
    if kind == "protein-iid":  # the Dayhoff table and the 10.0 cap
        a = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)[rng.integers(0, 20, (150, 300))]
        return a, oracle.PROTEIN, {}
    if kind == "protein-80":  # more residues than the tensor cores take: bit planes
        a = np.frombuffer(bytes(range(40, 120)), np.uint8)[rng.integers(0, 80, (150, 300))]
        a[rng.random(a.shape) < 0.05] = ord("-")
        return a, oracle.PROTEIN, {}
    if kind == "protein-wrap":  # L = 128: the reference's fast-path valid count
        return (synth.tree_protein(140, 128, seed=4, mean_branch=0.2), oracle.PROTEIN,
                {"compat_wrap": True})
    if kind == "dna-naive":
        s = synth.tree_dna(200, 400, seed=5, mean_branch=0.1)
        s[rng.random(s.shape) < 0.1] = ord("a")
        return s, oracle.DNA, {"fastdist": False}
    if kind == "dna-naive-full":
        s = synth.tree_dna(150, 300, seed=6, mean_branch=0.1)
        s[rng.random(s.shape) < 0.1] = ord("a")
        return s, oracle.DNA, {"fastdist": False, "full_rows": True}
    if kind == "tiny":
        return np.frombuffer(b"AC-T", np.uint8).reshape(1, 4).copy(), oracle.DNA, {}
    raise ValueError(kind)


KINDS = ["dna", "dna-saturated", "protein", "protein-iid", "protein-80", "protein-wrap",
         "dna-naive", "dna-naive-full", "tiny"]


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("model", ["kim", "jc"])
def test_double_matrix_against_oracle_and_float_matrix(ctx, kind, model):
    seqs, typ, opts = case(kind)
    aln = ctx.alignment(seqs, typ, **opts)
    got, gmax = ctx.distance_f64(aln, model)
    got = got.cpu().numpy()
    mat = ctx.distance(aln, model)
    flt = mat.to_numpy()
    mat.close()
    aln.close()
    naive = not opts.get("fastdist", True)
    full = opts.get("full_rows", False)
    c = oracle.counts(seqs, typ, naive=naive, full=full)
    m = oracle.JC if model == "jc" else oracle.KIMURA
    want, wmax = oracle.matrix_f64(c, seqs.shape[1], typ, m, naive=naive,
                                   compat_wrap=opts.get("compat_wrap", False), full=full)
    assert abs(gmax - wmax) <= 1e-12 * abs(wmax)
    err = np.abs(got - want)
    assert (err <= 1e-12 * np.abs(want)).all(), float((err / np.maximum(np.abs(want), 1e-300)).max())
    d = ulp_diff(got.astype(np.float32), flt)
    assert d.max() <= 1 and (d == 1).sum() <= max(2, 1e-6 * d.size)


def test_double_matrix_of_a_larger_tensor_core_alignment(ctx):
    from rapidnj_b200 import synth
    seqs = synth.tree_dna(2000, 3000, seed=11)
    aln = ctx.alignment(torch.from_numpy(seqs).cuda(), oracle.DNA)
    got, gmax = ctx.distance_f64(aln, "kim")
    out = torch.empty((2000, 2000), dtype=torch.float32, device="cuda")
    fmax = ctx.distance_into(aln, "kim", out, want_max=True)
    aln.close()
    d = ulp_diff(got.cpu().numpy().astype(np.float32), out.cpu().numpy())
    assert d.max() <= 1 and (d == 1).sum() <= max(2, 1e-6 * d.size)
    assert np.float32(gmax) == np.float32(fmax) or abs(np.float32(gmax) - fmax) <= 1e-6 * fmax
    # sampled pairs against the oracle's doubles
    rng = np.random.default_rng(2)
    rows = rng.integers(0, 2000, 40)
    sub = seqs[np.unique(rows)]
    c = oracle.counts(sub, oracle.DNA)
    want, _ = oracle.matrix_f64(c, sub.shape[1], oracle.DNA, oracle.KIMURA)
    g = got.cpu().numpy()[np.ix_(np.unique(rows), np.unique(rows))]
    off = ~np.eye(len(want), dtype=bool)
    assert (np.abs(g - want)[off] <= 1e-12 * np.abs(want)[off]).all()


def test_double_matrix_rejects_bad_arguments(ctx):
    from rapidnj_b200._native import RnjError
    seqs, typ, _ = case("dna")
    aln = ctx.alignment(seqs[:10], typ)
    small = torch.empty((10, 5), dtype=torch.float64, device="cuda")
    with pytest.raises(RnjError):
        ctx.distance_f64(aln, "kim", out=small)
    aln.close()
