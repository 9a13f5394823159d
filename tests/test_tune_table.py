"""The autotuner's bucket table (rnj_tune_get / _set / _clear / _save / _load and
RNJ_TUNE_CACHE): host logic only, no GPU needed."""
import os
import subprocess
import sys
import textwrap

import pytest

from rapidnj_b200 import api
from rapidnj_b200._native import RnjError

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(autouse=True)
def empty_table():
    api.tune_clear()
    yield
    api.tune_clear()


def test_set_get_and_buckets():
    assert api.tune_get(1000, 5000, "dna") is None
    api.tune_set(1000, 5000, "dna", dna_kernel=1, ksplit=4, tile_band=8, transform_ctas=3,
                 stream_band=16)
    p = api.tune_get(1000, 5000, "dna")
    assert (p.dna_kernel, p.ksplit, p.tile_band, p.transform_ctas, p.stream_band) == (1, 4, 8, 3, 16)
    # same bucket: floor(log2 n) = 9, floor(log2 L) = 12
    assert api.tune_get(512, 4096, "dna").ksplit == 4
    assert api.tune_get(1023, 8191, "dna").ksplit == 4
    # other buckets: n, L, alphabet, rules
    assert api.tune_get(1024, 5000, "dna") is None
    assert api.tune_get(1000, 8192, "dna") is None
    assert api.tune_get(1000, 5000, "protein") is None
    assert api.tune_get(1000, 5000, "dna", fastdist=False) is None


@pytest.mark.parametrize("field,value", [("dna_kernel", 2), ("ksplit", -1), ("ksplit", 65),
                                         ("transform_ctas", 6), ("tile_band", -3)])
def test_out_of_range_rejected(field, value):
    with pytest.raises(RnjError):
        api.tune_set(100, 100, "dna", **{field: value})


def test_save_load_roundtrip(tmp_path):
    api.tune_set(10000, 10000, "dna", tile_band=12, transform_ctas=5, stream_band=16, ms=1.25)
    api.tune_set(300, 6000, "protein", ksplit=8, ms=0.5)
    path = str(tmp_path / "tune.txt")
    api.tune_save(path)
    text = open(path).read().splitlines()
    assert text[0].startswith("#") and len(text) == 3
    api.tune_clear()
    assert api.tune_get(300, 6000, "protein") is None
    api.tune_load(path)
    assert api.tune_get(300, 6000, "protein").ksplit == 8
    d = api.tune_get(10000, 10000, "dna")
    assert (d.tile_band, d.stream_band) == (12, 16) and abs(d.ms - 1.25) < 1e-4


def test_load_rejects_malformed(tmp_path):
    path = tmp_path / "bad.txt"
    path.write_text("dna 0 13 13 0 1 12 5\n")  # too few fields
    with pytest.raises(RnjError):
        api.tune_load(str(path))
    path.write_text("rna 0 13 13 0 1 12 5 16 1.0\n")
    with pytest.raises(RnjError):
        api.tune_load(str(path))
    with pytest.raises(RnjError):
        api.tune_load(str(tmp_path / "missing.txt"))


def test_env_cache_is_read_on_first_use(tmp_path):
    path = tmp_path / "cache.txt"
    path.write_text("# table\nprotein 0 8 12 0 4 0 0 0 0.7500\n")
    code = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {ROOT!r})
        from rapidnj_b200 import api
        p = api.tune_get(300, 5000, "protein")
        print(p.ksplit)
    """)
    env = dict(os.environ, RNJ_TUNE_CACHE=str(path))
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                         check=True)
    assert out.stdout.strip() == "4"


def test_epilogue_choice_and_earlier_file_form(tmp_path):
    api.tune_set(10000, 10000, "dna", tc_epilogue=1, ms=1.0)
    assert api.tune_get(10000, 10000, "dna").tc_epilogue == 1
    with pytest.raises(RnjError):
        api.tune_set(100, 100, "dna", tc_epilogue=2)
    path = str(tmp_path / "t.txt")
    api.tune_save(path)
    api.tune_clear()
    api.tune_load(path)
    assert api.tune_get(10000, 10000, "dna").tc_epilogue == 1
    # a table written before the epilogue field existed: ten fields, ms last
    old = tmp_path / "v1.txt"
    old.write_text("# v1\ndna 0 13 13 0 1 12 5 16 1.2500\n")
    api.tune_clear()
    api.tune_load(str(old))
    p = api.tune_get(10000, 10000, "dna")
    assert (p.tile_band, p.stream_band, p.tc_epilogue) == (12, 16, 0) and abs(p.ms - 1.25) < 1e-4


def test_ring_depths_and_eleven_field_form(tmp_path):
    api.tune_set(10000, 10000, "dna", tc_stages=4, pop_stages=3, ms=1.0)
    p = api.tune_get(10000, 10000, "dna")
    assert (p.tc_stages, p.pop_stages) == (4, 3)
    for field, value in (("tc_stages", 8), ("tc_stages", -1), ("pop_stages", 5)):
        with pytest.raises(RnjError):
            api.tune_set(100, 100, "dna", **{field: value})
    path = str(tmp_path / "t.txt")
    api.tune_save(path)
    line = open(path).read().splitlines()[1].split()
    assert len(line) == 13 and line[10:12] == ["4", "3"]
    api.tune_clear()
    api.tune_load(path)
    assert api.tune_get(10000, 10000, "dna").tc_stages == 4
    # the form with tc_epilogue but without the ring depths: eleven fields
    old = tmp_path / "v2.txt"
    old.write_text("# v2\nprotein 0 12 10 0 2 8 5 0 1 0.5000\n")
    api.tune_clear()
    api.tune_load(str(old))
    p = api.tune_get(5000, 1500, "protein")
    assert (p.ksplit, p.tile_band, p.tc_epilogue, p.tc_stages, p.pop_stages) == (2, 8, 1, 0, 0)
    # a fractional integer field is malformed
    old.write_text("dna 0 13 13 0 1.5 12 5 16 1 0 0 1.0\n")
    with pytest.raises(RnjError):
        api.tune_load(str(old))


def test_shipped_table_beside_the_library(tmp_path):
    # A copy of the library with a tune_b200.txt beside it reads that table at
    # its first lookup; RNJ_NO_TUNE_TABLE turns it off, RNJ_TUNE_CACHE wins.
    import shutil
    lib = os.path.join(ROOT, "rapidnj_b200", "librnjgpu.so")
    shutil.copy(lib, tmp_path / "librnjgpu.so")
    (tmp_path / "tune_b200.txt").write_text("# shipped\ndna 0 13 13 0 1 8 0 0 0 5 0 1.0\n")
    other = tmp_path / "other.txt"
    other.write_text("dna 0 13 13 0 1 24 0 0 0 3 0 1.0\n")
    code = textwrap.dedent(f"""
        import ctypes
        lib = ctypes.CDLL({str(tmp_path / "librnjgpu.so")!r})
        p = (ctypes.c_int * 9)()
        rc = lib.rnj_tune_get(10000, 10000, 0, 1, p)
        print(rc, p[2], p[6])
    """)

    def run(**env):
        e = {k: v for k, v in os.environ.items()
             if k not in ("RNJ_TUNE_CACHE", "RNJ_NO_TUNE_TABLE")}
        e.update(env)
        out = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True,
                             text=True, check=True)
        return out.stdout.split()

    assert run() == ["0", "8", "5"]
    assert run(RNJ_NO_TUNE_TABLE="1")[0] != "0"
    assert run(RNJ_TUNE_CACHE=str(other)) == ["0", "24", "3"]
