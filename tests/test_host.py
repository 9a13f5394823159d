"""Host-side checks that need no GPU: the C-ABI library loads and exports every
declared symbol, the alignment reader and the "-o m" writer reproduce the
reference byte for byte, and the synthetic workloads are seeded."""
import os
import re
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, golden_files, load_golden

HEADER = os.path.join(ROOT, "include", "rnj.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rnj_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_all_declared_symbols():
    from rapidnj_b200 import _native
    lib = _native.lib()
    missing = [s for s in declared_symbols() if getattr(lib, s, None) is None]
    assert not missing, missing
    assert len(declared_symbols()) >= 25


def test_version_string():
    from rapidnj_b200 import api
    assert "sm_100a" in api.version()


def test_context_without_gpu_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from rapidnj_b200 import api, RnjError
    with pytest.raises(RnjError):
        api.Context(0)


def test_detect_type_matches_reference_rule():
    from rapidnj_b200 import api
    assert api.detect_type(b"ACGTN-acgtun") == 0
    assert api.detect_type(b"ACGTE") == 1
    assert api.detect_type(b"ACGT*?.-123") == 0


@pytest.mark.parametrize("path", [p for p in golden_files() if "fixture" in p or "stockholm" in p],
                         ids=lambda p: p.split("/")[-1])
def test_reader_matches_reference_parse(path, tmp_path):
    from rapidnj_b200 import api
    g = load_golden(path)
    if "sth_text" in g:
        f = tmp_path / "a.sth"
        f.write_bytes(bytes(g["sth_text"]))
        names, chars, t = api.read_alignment(str(f), "sth")
    else:
        f = tmp_path / "a.fa"
        f.write_bytes(bytes(g["fa_text"]))
        names, chars, t = api.read_alignment(str(f))
    assert np.array_equal(chars, g["chars"])
    assert names[: len(g["names"])] == g["names"]
    if g["type_arg"] == "auto":
        assert t == int(g["ref_type"])


def test_reader_rejects_ragged_and_truncated(tmp_path):
    from rapidnj_b200 import api, RnjError
    f = tmp_path / "bad.fa"
    f.write_bytes(b">a\nACGT\n>b\nACG\n")
    with pytest.raises(RnjError, match="length"):
        api.read_alignment(str(f))
    s = tmp_path / "bad.sth"
    s.write_bytes(b"# STOCKHOLM 1.0\na ACGT\nb ACGT\n")
    with pytest.raises(RnjError, match="//"):
        api.read_alignment(str(s))
    with pytest.raises(RnjError):
        api.read_alignment(str(tmp_path / "missing.fa"))


def test_reader_fasta_rules(tmp_path):
    """';' comment lines, multi-line sequences, bytes <= 32 dropped, CRLF."""
    from rapidnj_b200 import api
    f = tmp_path / "x.fasta"
    f.write_bytes(b";comment\r\n>one two\r\nAC GT\r\nAC\r\n>three\nACGT\tAC\n")
    names, chars, t = api.read_alignment(str(f))
    assert names == ["one two", "three"]
    assert chars.tobytes() == b"ACGTACACGTAC"


def test_reader_fasta_name_terminators(tmp_path):
    """A name ends at the first byte <= 31 (or >= 128); the rest of its line is
    read as if a line began there, as the reference's character loop
    (dataloaderFasta.hpp:78-133) reads it: a ';' there starts a comment, a '>'
    another name; sequence bytes >= 128 are dropped like control bytes."""
    from rapidnj_b200 import api
    f = tmp_path / "t.fa"
    f.write_bytes(b">a\t;comment\nACGT\n>b\r\nAC\x80GT\n>c\t>d\nACGT")
    names, chars, t = api.read_alignment(str(f))
    assert names == ["a", "b", "c", "d"]
    assert chars.shape == (3, 4) and chars.tobytes() == b"ACGTACGTACGT"


@pytest.mark.parametrize("fixture", ["fixture_LGT_70", "fixture_PF15224_full"])
@pytest.mark.parametrize("model", ["jc", "kim"])
def test_matrix_text_matches_reference_binary(fixture, model, tmp_path):
    """The "-o m" writer, given the reference's own matrix, prints the reference's text."""
    from rapidnj_b200 import api
    g = load_golden(os.path.join(GOLDEN, fixture + ".npz"))
    out = tmp_path / "m.txt"
    api.write_matrix_text(str(out), g["names"], g[f"{model}_fast"], threads=3)
    assert out.read_bytes() == bytes(g[f"text_{model}"])


def test_synthetic_workloads_are_seeded():
    from rapidnj_b200 import synth
    a = synth.tree_dna(64, 300, seed=5)
    b = synth.tree_dna(64, 300, seed=5)
    assert np.array_equal(a, b)
    assert set(np.unique(a).tobytes()) <= set(b"ACGT-")
    p = synth.tree_protein(40, 200, seed=1)
    assert abs((p == ord("-")).mean() - 0.08) < 0.03
    d = synth.iid_dna(100, 2000, seed=0)
    assert abs((d == ord("-")).mean() - 0.05) < 0.01
    mix = synth.batch_mix(4, seed=2)
    assert len(mix) == 4 and all(k in ("dna", "protein") for k, _ in mix)
