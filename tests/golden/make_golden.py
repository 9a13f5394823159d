"""Generates tests/golden/*.npz from the reference itself.

Runs only where the rapidNJ source tree is present (it builds and calls
oracle/_ref/ref_harness and oracle/_ref/rapidnj, compiled from the reference
sources by oracle/Makefile).  The outputs are committed; the tests only read
them, so nothing here runs on the GPU box.

Cases
-----
* the reference's own fixtures: test_data/LGT_70.fa (DNA, 68 x 1302) and
  test_data/PF15224_full.fa (protein, 41 x 86)
* crafted DNA alignments at L in {1, 31, 32, 33, 63, 64, 65, 127, 128, 129, 383,
  384, 385}: all-gap rows, identical rows, lower case, U/N/IUPAC letters and
  other gap bytes, random and saturated pairs
* crafted protein alignments at L in {1, 15, 16, 17, 127, 128, 129, 255, 256,
  257, 300}: the gap set (- . X x z Z b B J j ?), lower case, saturated pairs
* a protein alignment whose pairs walk p = 0.700 .. 1.000 through the Dayhoff
  table range
* a Stockholm copy of one crafted DNA case (parser parity)

For each case the reference provides: per-pair counts from its estimators (fast
bit-string path and naive -f path, upper triangle and full rows), and the
post-processed float matrices from its JCdistance / KimuraDistance drivers (fast
and naive; one disk-matrix run).  For the two fixtures also the exact "-o m" text
of the reference binary.

Usage: python tests/golden/make_golden.py   (from the repository root)
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402  (test infrastructure)

REF = oracle.reference_tree()  # $RNJ_REFERENCE, else a `reference` folder beside the repo
OUT = os.path.join(ROOT, "tests", "golden")


def parse_fasta_bytes(path):
    """Names and sequence bytes with the reference FASTA rules
    (dataloaderFasta.hpp:78-133): ';' lines skipped, '>' starts a name of bytes
    > 31, other lines contribute their bytes > 32, end of file reads as '\\n'."""
    data = open(path, "rb").read()
    pos, names, seqs, cur = 0, [], [], bytearray()

    def nxt():
        nonlocal pos
        if pos < len(data):
            pos += 1
            return data[pos - 1], False
        return 10, True

    while True:
        c, eof = nxt()
        if eof:
            break
        if c == ord(";"):
            while c != 10:
                c, _ = nxt()
        elif c == ord(">"):
            if cur:
                seqs.append(bytes(cur))
                cur = bytearray()
            c, _ = nxt()
            name = bytearray()
            while c > 31:
                name.append(c)
                c, _ = nxt()
            names.append(name.decode("latin-1"))
        else:
            while c != 10:
                if c > 32:
                    cur.append(c)
                c, _ = nxt()
    if cur:
        seqs.append(bytes(cur))
    L = len(seqs[0])
    assert all(len(s) == L for s in seqs)
    return names, np.frombuffer(b"".join(seqs), dtype=np.uint8).reshape(len(seqs), L)


def write_fasta(path, names, seqs):
    with open(path, "wb") as f:
        for nm, s in zip(names, seqs):
            f.write(b">" + nm.encode() + b"\n" + s.tobytes() + b"\n")


def write_stockholm(path, names, seqs):
    with open(path, "wb") as f:
        f.write(b"# STOCKHOLM 1.0\n#=GF ID crafted\n")
        for nm, s in zip(names, seqs):
            f.write(nm.encode() + b"   " + s.tobytes() + b"\n")
        f.write(b"//\n")


def reference_outputs(path, fmt, t, with_text=False):
    out = {}
    c, L, typ = oracle.ref_counts(path, fmt, t, fastdist=True)
    out["ref_type"] = np.int32(typ)
    out["counts_fast"] = c
    out["counts_naive"], _, _ = oracle.ref_counts(path, fmt, t, fastdist=False)
    out["counts_naive_full"], _, _ = oracle.ref_counts(path, fmt, t, fastdist=False, full=True)
    for model in ("jc", "kim"):
        m, _ = oracle.ref_matrix(path, model, fmt, t, fastdist=True, threads=3)
        out[f"{model}_fast"] = m
        m, _ = oracle.ref_matrix(path, model, fmt, t, fastdist=False, threads=2)
        out[f"{model}_naive"] = m
    m, _ = oracle.ref_matrix(path, "kim", fmt, t, fastdist=True, threads=2, disk=True)
    out["kim_fast_disk"] = m
    m, _ = oracle.ref_matrix(path, "kim", fmt, t, fastdist=False, threads=2, disk=True)
    out["kim_naive_disk"] = m
    if with_text:
        for model in ("jc", "kim"):
            p = subprocess.run([oracle.REF_RAPIDNJ, path, "-i", fmt, "-o", "m", "-a", model, "-c", "2"],
                               check=True, capture_output=True)
            out[f"text_{model}"] = np.frombuffer(p.stdout, dtype=np.uint8)
    return out


def crafted_dna(L, rng):
    alphabet = np.frombuffer(b"ACGT", dtype=np.uint8)
    base = alphabet[rng.integers(0, 4, L)]
    rows = [base.copy()]                                    # row 0: plain ACGT (type detection)
    rows.append(base.copy())                                # identical
    r = base.copy(); r[rng.random(L) < 0.1] = ord("-"); rows.append(r)
    rows.append(alphabet[rng.integers(0, 4, L)])            # unrelated (saturates often)
    rows.append(np.full(L, ord("-"), np.uint8))             # all gaps
    rows.append(np.frombuffer(base.tobytes().lower(), np.uint8).copy())  # lower case
    mixed = np.frombuffer(b"ACGTacgtUuNnRY.-?*", np.uint8)
    rows.append(mixed[rng.integers(0, mixed.size, L)])      # ambiguity / gap bytes
    comp = {65: 84, 84: 65, 67: 71, 71: 67}
    rows.append(np.array([comp[int(x)] for x in base], np.uint8))  # transversions everywhere
    ts = {65: 71, 71: 65, 67: 84, 84: 67}
    r = base.copy(); m = rng.random(L) < 0.4
    r[m] = [ts[int(x)] for x in base[m]]; rows.append(r)    # heavy transitions
    r = base.copy(); m = rng.random(L) < 0.05
    r[m] = alphabet[rng.integers(0, 4, int(m.sum()))]; rows.append(r)
    rows.append(np.full(L, ord("A"), np.uint8))
    rows.append(np.full(L, ord("U"), np.uint8))
    return np.stack(rows)


def crafted_protein(L, rng):
    amino = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", np.uint8)
    base = amino[rng.integers(0, 20, L)]
    base[0] = ord("E")  # unambiguous protein letter in row 0
    rows = [base.copy(), base.copy()]
    r = base.copy(); r[rng.random(L) < 0.08] = ord("-"); rows.append(r)
    rows.append(amino[rng.integers(0, 20, L)])
    rows.append(np.full(L, ord("-"), np.uint8))
    gapset = np.frombuffer(b"-.XxzZbBJj?", np.uint8)
    r = base.copy(); m = rng.random(L) < 0.3
    r[m] = gapset[rng.integers(0, gapset.size, int(m.sum()))]; rows.append(r)
    rows.append(np.frombuffer(base.tobytes().lower(), np.uint8).copy())
    for frac in (0.2, 0.5, 0.8):
        r = base.copy(); m = rng.random(L) < frac
        r[m] = amino[rng.integers(0, 20, int(m.sum()))]; rows.append(r)
    other = np.frombuffer(b"BOUZ*#acdefghik", np.uint8)
    rows.append(other[rng.integers(0, other.size, L)])
    rows.append(np.full(L, ord("W"), np.uint8))
    return np.stack(rows)


def pam_walk(rng, L=1000):
    amino = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", np.uint8)
    base = amino[rng.integers(0, 20, L)]
    rows = [base]
    for k in list(range(700, 1001, 7)) + [749, 750, 751, 929, 930, 931, 932]:
        r = base.copy()
        pos = rng.choice(L, k, replace=False)
        shift = rng.integers(1, 20, k)
        idx = np.searchsorted(amino, r[pos], sorter=np.argsort(amino))
        r[pos] = amino[np.argsort(amino)[(idx + shift) % 20]]
        rows.append(r)
    return np.stack(rows)


def save(name, names, seqs, outputs, fmt="fa", t="auto"):
    d = dict(outputs)
    d["chars"] = seqs
    d["names"] = np.frombuffer("\n".join(names).encode(), dtype=np.uint8)
    d["fmt"] = np.frombuffer(fmt.encode(), np.uint8)
    d["type_arg"] = np.frombuffer(t.encode(), np.uint8)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)


def main():
    if REF is None:
        sys.exit("the rapidNJ source tree was not found: set RNJ_REFERENCE")
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", "ref", f"REF={REF}"],
                   check=True)
    rng = np.random.default_rng(20240611)
    with tempfile.TemporaryDirectory() as td:
        for fx in ("LGT_70.fa", "PF15224_full.fa"):
            path = os.path.join(REF, "test_data", fx)
            names, seqs = parse_fasta_bytes(path)
            out = reference_outputs(path, "fa", "auto", with_text=True)
            out["fa_text"] = np.frombuffer(open(path, "rb").read(), np.uint8)
            save("fixture_" + fx.split(".")[0], names, seqs, out)
        for L in (1, 31, 32, 33, 63, 64, 65, 127, 128, 129, 383, 384, 385):
            seqs = crafted_dna(L, rng)
            names = [f"d{i}" for i in range(len(seqs))]
            path = os.path.join(td, f"dna_{L}.fa")
            write_fasta(path, names, seqs)
            save(f"dna_L{L}", names, seqs, reference_outputs(path, "fa", "d"), t="d")
        for L in (1, 15, 16, 17, 127, 128, 129, 255, 256, 257, 300):
            seqs = crafted_protein(L, rng)
            names = [f"p{i}" for i in range(len(seqs))]
            path = os.path.join(td, f"prot_{L}.fa")
            write_fasta(path, names, seqs)
            save(f"protein_L{L}", names, seqs, reference_outputs(path, "fa", "p"), t="p")
        seqs = pam_walk(rng)
        names = [f"w{i}" for i in range(len(seqs))]
        path = os.path.join(td, "pam.fa")
        write_fasta(path, names, seqs)
        save("protein_pam_walk", names, seqs, reference_outputs(path, "fa", "p"), t="p")
        seqs = crafted_dna(200, rng)
        names = [f"sth{i}" for i in range(len(seqs))]
        path = os.path.join(td, "dna.sth")
        write_stockholm(path, names, seqs)
        out = reference_outputs(path, "sth", "d")
        out["sth_text"] = np.frombuffer(open(path, "rb").read(), np.uint8)
        save("stockholm_dna", names, seqs, out, fmt="sth", t="d")
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
