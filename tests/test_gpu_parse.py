"""rnj_msa_read_device: the FASTA file parsed on the device (newline compaction,
line kinds, per-sequence scan, byte compaction).  Every file must give exactly
the host reader's names, bytes and type (rnj_msa_read, pinned to the reference's
own loader by the golden fixtures), including the inputs the device path hands
to the host rules, and the same error for sequences of different lengths."""
import os

import numpy as np
import pytest

from conftest import golden_files, load_golden
from rapidnj_b200 import api, synth
from rapidnj_b200._native import RnjError

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def same_as_host(ctx, path, fmt=None):
    hn, hc, ht = api.read_alignment(path, fmt)
    dn, dc, dt = ctx.read_alignment_device(path, fmt)
    assert dn == hn
    assert dt == ht
    assert np.array_equal(dc.cpu().numpy(), hc)
    return dn, dc, dt


def write(path, data: bytes):
    with open(path, "wb") as f:
        f.write(data)
    return str(path)


@pytest.mark.parametrize("gpath", [p for p in golden_files()],
                         ids=[os.path.basename(p)[:-4] for p in golden_files()])
def test_golden_fixtures(ctx, tmp_path, gpath):
    g = load_golden(gpath)
    if g["fmt"] != "fa":
        pytest.skip("Stockholm fixture (covered below)")
    if "fa_text" in g:
        path = write(tmp_path / "f.fa", bytes(g["fa_text"]))
        same_as_host(ctx, path)
    for width in (0, 7, 60):
        p = tmp_path / f"w{width}.fa"
        synth.write_fasta(str(p), g["chars"], names=g["names"][:g["chars"].shape[0]], width=width)
        same_as_host(ctx, str(p))


@pytest.mark.parametrize("n,L,width", [(300, 1000, 0), (1000, 2000, 60), (2500, 777, 61),
                                       (64, 70000, 80), (5000, 300, 1)])
def test_layouts(ctx, tmp_path, n, L, width):
    s = synth.tree_dna(n, L, seed=n + L, mean_branch=0.05)
    p = str(tmp_path / "a.fa")
    synth.write_fasta(p, s, width=width)
    names, chars, t = same_as_host(ctx, p)
    assert np.array_equal(chars.cpu().numpy(), s) and len(names) == n


def test_protein_and_line_endings(ctx, tmp_path):
    s = synth.tree_protein(400, 900, seed=3)
    rows = [b">p%d descr\r\n" % i + b"\r\n".join(s[i, k:k + 50].tobytes() for k in range(0, 900, 50))
            + b"\r\n" for i in range(400)]
    p = write(tmp_path / "crlf.fa", b"".join(rows))
    names, chars, t = same_as_host(ctx, p)
    assert t == 1 and names[0] == "p0 descr"


def test_comments_blank_lines_spaces_high_bytes(ctx, tmp_path):
    data = (b";comment line\n>a\nAC GT\tAC\n\n;another\nGG\x80TT\n>b x\n  ACGTACGG\nTT\n"
            b">c\nACGT\nACGGTT")  # no newline at the end
    same_as_host(ctx, write(tmp_path / "c.fa", data))


@pytest.mark.parametrize("data", [
    b">a\tdesc ACGT\nACGT\n>b\tx\nACGTACGT\n",     # a name ended by a tab: the rest is data
    b"ACGT\n>a\nACGT\n>b\nACGT\n",                 # data before the first name
    b">a\nACGT\n>empty\n>b\nACGT\n",               # a name without data
    b"ACGTACGT\nACGT\n",                           # no name at all
    b">a\x01b\nACGT\n>c\nACGT\n",                  # a control byte inside a name
    b">a\xc3\xa9\nACGT\n>b\nACGT\n",               # bytes >= 128 end a name
    b">a\n>b\nACGT\n>c\nACGT\n",                   # two names in a row
])
def test_host_rule_inputs(ctx, tmp_path, data):
    p = write(tmp_path / "q.fa", data)
    try:
        hn, hc, ht = api.read_alignment(p)
    except RnjError as e:
        with pytest.raises(RnjError) as d:
            ctx.read_alignment_device(p)
        assert str(d.value) == str(e)
        return
    same_as_host(ctx, p)


def test_length_mismatch_error(ctx, tmp_path):
    p = write(tmp_path / "bad.fa", b">a\nACGT\n>b\nACGTA\n>c\nACG\n")
    with pytest.raises(RnjError) as h:
        api.read_alignment(p)
    with pytest.raises(RnjError) as d:
        ctx.read_alignment_device(p)
    assert str(d.value) == str(h.value)
    assert "Sequence 1 has length 5" in str(d.value)


def test_stockholm_goes_through_host_rules(ctx, tmp_path):
    seen = 0
    for gpath in golden_files():
        g = load_golden(gpath)
        if g["fmt"] == "sth":
            same_as_host(ctx, write(tmp_path / "a.sth", bytes(g["sth_text"])))
            seen += 1
    assert seen >= 1


def test_missing_file(ctx, tmp_path):
    with pytest.raises(RnjError, match="Could not read file"):
        ctx.read_alignment_device(str(tmp_path / "none.fa"))


def test_parse_then_distance(ctx, tmp_path):
    # file -> device bytes -> distances, equal to the host-read path
    s = synth.tree_dna(700, 1500, seed=4)
    p = str(tmp_path / "d.fa")
    synth.write_fasta(p, s, width=60)
    names, chars, t = ctx.read_alignment_device(p)
    aln = ctx.alignment(chars, t)
    out = torch.empty((700, 700), dtype=torch.float32, device="cuda")
    ctx.distance_into(aln, "kim", out)
    aln.close()
    ref = ctx.distance(ctx.alignment(s, 0), "kim").to_numpy()
    assert np.array_equal(out.cpu().numpy().view(np.int32), ref.view(np.int32))


def test_repeated_reads_reuse_the_buffer(ctx, tmp_path):
    a = synth.tree_dna(200, 300, seed=1)
    b = synth.tree_dna(900, 4000, seed=2)
    pa, pb = str(tmp_path / "a.fa"), str(tmp_path / "b.fa")
    synth.write_fasta(pa, a, width=60)
    synth.write_fasta(pb, b)
    for p in (pa, pb, pa):
        same_as_host(ctx, p)
