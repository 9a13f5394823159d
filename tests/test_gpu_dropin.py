"""The C++ drop-in inside rapidNJ itself: the reference's unchanged CLI linked
with our JCdistance / KimuraDistance (oracle/_ref/rapidnj_b200) against the
unchanged reference binary (oracle/_ref/rapidnj), on the same inputs.  The
distance matrices ("-o m" text) and the trees its join loops build from them
must be byte-identical, through the fast and naive (-f) estimators, the
bootstrap loop (-b, main.cpp:519-532) and the disk-backed matrix (-d).

Both binaries are built from the reference sources where they lie (oracle/Makefile
targets ref and dropin); the tests skip when they are absent."""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

pytestmark = pytest.mark.gpu

REF = os.path.join(ROOT, "oracle", "_ref", "rapidnj")
DROPIN = os.path.join(ROOT, "oracle", "_ref", "rapidnj_b200")


def need_binaries():
    if not (os.path.exists(REF) and os.path.exists(DROPIN)):
        pytest.skip("reference CLI builds (oracle/_ref) not present")


def fixture(tmp_path, name):
    z = np.load(os.path.join(GOLDEN, f"fixture_{name}.npz"))
    p = tmp_path / f"{name}.fa"
    p.write_bytes(bytes(z["fa_text"]))
    return str(p)


def run(binary, args, tmp_path, env=None):
    r = subprocess.run([binary] + args, capture_output=True, timeout=600, cwd=str(tmp_path),
                       env=dict(os.environ, **(env or {})))
    assert r.returncode == 0, (binary, args, r.stderr.decode()[-2000:])
    return r.stdout


def same_output(args, tmp_path, env=None):
    need_binaries()
    want = run(REF, args, tmp_path)
    got = run(DROPIN, args, tmp_path, env)
    assert len(want) > 0
    assert got == want, f"output differs for {args}"


@pytest.mark.parametrize("name", ["LGT_70", "PF15224_full"])
@pytest.mark.parametrize("model", ["jc", "kim"])
@pytest.mark.parametrize("fast", [True, False])
def test_distance_matrix_text(tmp_path, name, model, fast):
    args = [fixture(tmp_path, name), "-o", "m", "-a", model] + ([] if fast else ["-f"])
    same_output(args, tmp_path)


@pytest.mark.parametrize("name", ["LGT_70", "PF15224_full"])
def test_tree(tmp_path, name):
    same_output([fixture(tmp_path, name), "-a", "kim", "-c", "4"], tmp_path)


def test_bootstrap_trees(tmp_path):
    same_output([fixture(tmp_path, "LGT_70"), "-a", "kim", "-b", "5", "-c", "2"], tmp_path)


@pytest.mark.parametrize("fast", [True, False])
def test_disk_matrix_tree(tmp_path, fast):
    cache = tmp_path / "cache"
    cache.mkdir()
    args = [fixture(tmp_path, "LGT_70"), "-a", "kim", "-d", str(cache)] + ([] if fast else ["-f"])
    same_output(args, tmp_path)


def test_synthetic_multi_tile(tmp_path):
    """600 tree-evolved DNA sequences (5 x 5 tiles of pairs), both models."""
    from rapidnj_b200 import synth
    p = tmp_path / "syn.fa"
    synth.write_fasta(str(p), synth.tree_dna(600, 1500, seed=21, mean_branch=0.05))
    for model in ("jc", "kim"):
        same_output([str(p), "-o", "m", "-a", model], tmp_path)
    same_output([str(p), "-a", "kim"], tmp_path)


# A device-matrix budget far below the n x n floats: the drop-in computes the
# rows in bands of 128 (rnj_distance_rows, two band buffers on the device) and
# hands them to the disk matrix or to the row arrays, post-processing the rows
# with saturated pairs as the reference does.
SMALL_BUDGET = {"RNJ_DEVICE_MATRIX_BUDGET": "100000"}


def synthetic_files(tmp_path):
    from rapidnj_b200 import synth
    p = tmp_path / "syn.fa"
    synth.write_fasta(str(p), synth.tree_dna(600, 1500, seed=21, mean_branch=0.05))
    rng = np.random.default_rng(4)
    q = tmp_path / "sat.fa"  # unrelated short sequences: many saturated pairs
    synth.write_fasta(str(q), np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (300, 40))])
    return str(p), str(q)


@pytest.mark.parametrize("fast", [True, False])
def test_matrix_beyond_device_budget_disk_mode(tmp_path, fast):
    """-d: the disk-matrix tree and -o m text of matrices larger than the budget."""
    syn, sat = synthetic_files(tmp_path)
    cache = tmp_path / "cache"
    cache.mkdir()
    f = [] if fast else ["-f"]
    for path in (syn, sat):
        same_output([path, "-a", "kim", "-d", str(cache)] + f, tmp_path, SMALL_BUDGET)
        same_output([path, "-o", "m", "-a", "jc", "-d", str(cache)] + f, tmp_path, SMALL_BUDGET)


def test_matrix_beyond_device_budget_in_memory(tmp_path):
    """No disk matrix: the banded rows fill rapidNJ's in-memory rows."""
    syn, sat = synthetic_files(tmp_path)
    for path in (syn, sat):
        same_output([path, "-o", "m", "-a", "kim"], tmp_path, SMALL_BUDGET)
    same_output([syn, "-a", "kim"], tmp_path, SMALL_BUDGET)
    same_output([fixture(tmp_path, "PF15224_full"), "-o", "m", "-a", "kim"], tmp_path,
                SMALL_BUDGET)


def test_dropin_fails_loudly_on_a_bad_device(tmp_path):
    need_binaries()
    env = dict(os.environ, RNJ_DEVICE="4096")
    r = subprocess.run([DROPIN, fixture(tmp_path, "LGT_70"), "-o", "m"], capture_output=True,
                       timeout=120, env=env)
    assert r.returncode == 1 and b"ERROR" in r.stderr


# --------------------------------------------- the standalone program (rnj-b200)

CLI = os.path.join(ROOT, "rapidnj_b200", "rnj-b200")


@pytest.mark.parametrize("name", ["LGT_70", "PF15224_full"])
@pytest.mark.parametrize("model", ["jc", "kim"])
def test_cli_matches_reference_text(tmp_path, name, model):
    """rnj-b200 -o m against the reference's own "-o m" output kept in the goldens."""
    if not os.path.exists(CLI):
        pytest.skip("rnj-b200 not built")
    z = np.load(os.path.join(GOLDEN, f"fixture_{name}.npz"))
    got = run(CLI, [fixture(tmp_path, name), "-o", "m", "-a", model, "-c", "4"], tmp_path)
    assert got == bytes(z[f"text_{model}"])
    out = tmp_path / "m.txt"
    run(CLI, [fixture(tmp_path, name), "-a", model, "-x", str(out)], tmp_path)
    assert out.read_bytes() == bytes(z[f"text_{model}"])
