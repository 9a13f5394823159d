"""Python face of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of bench.py
import this module, and only as the checker.  The product path never does.

* ``counts`` / ``matrix`` call the C restatement in ``liborc.so``
  (``rnj_oracle.c``; parity pinned against the reference's own outputs by
  tests/test_oracle_golden.py).
* ``ref_counts`` / ``ref_matrix`` run the reference's own code through
  ``_ref/ref_harness`` (built from the reference sources by this folder's
  Makefile) when it is present.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liborc.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_HARNESS = os.path.join(REF_DIR, "ref_harness")
REF_RAPIDNJ = os.path.join(REF_DIR, "rapidnj")

DNA, PROTEIN = 0, 1
JC, KIMURA = 0, 1

_lib = None


def build() -> None:
    """Compile liborc.so (and the reference harness when the reference tree is
    present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    if os.path.isdir(os.environ.get("RNJ_REFERENCE", "/root/reference")):
        subprocess.run(["make", "-s", "-C", HERE, "ref",
                        "REF=" + os.environ.get("RNJ_REFERENCE", "/root/reference")], check=True)
        if os.path.exists(os.path.join(HERE, "..", "rapidnj_b200", "librnjgpu.so")):
            subprocess.run(["make", "-s", "-C", HERE, "dropin",
                            "REF=" + os.environ.get("RNJ_REFERENCE", "/root/reference")],
                           check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
        f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
        L.orc_counts.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, u32p]
        L.orc_counts.restype = None
        L.orc_matrix.argtypes = [u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_int, f32p]
        L.orc_matrix.restype = ctypes.c_float
        L.orc_matrix_full.argtypes = L.orc_matrix.argtypes
        L.orc_matrix_full.restype = ctypes.c_float
        L.orc_raw_distances.argtypes = [u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        f32p]
        L.orc_raw_distances.restype = None
        L.orc_detect_type.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.orc_detect_type.restype = ctypes.c_int
        L.orc_jc.argtypes = [ctypes.c_uint64] * 3 + [ctypes.c_int]
        L.orc_jc.restype = ctypes.c_float
        L.orc_k2p.argtypes = [ctypes.c_uint64] * 3
        L.orc_k2p.restype = ctypes.c_float
        L.orc_kimura_protein.argtypes = [ctypes.c_uint64] * 2
        L.orc_kimura_protein.restype = ctypes.c_float
        L.orc_protein_fast_valid.argtypes = [ctypes.c_uint64, ctypes.c_int]
        L.orc_protein_fast_valid.restype = ctypes.c_uint64
        L.orc_pam_value.argtypes = [ctypes.c_int]
        L.orc_pam_value.restype = ctypes.c_int
        _lib = L
    return _lib


def detect_type(seqs: np.ndarray) -> int:
    row = np.ascontiguousarray(seqs[0], dtype=np.uint8)
    return lib().orc_detect_type(row.tobytes(), row.size)


def counts(seqs: np.ndarray, type_: int, naive: bool = False, full: bool = False) -> np.ndarray:
    """(n, n, 3) uint32: {ts, tv, valid} (DNA) or {mismatch, 0, valid} (protein)
    for j > i (every pair when ``full``)."""
    s = np.ascontiguousarray(seqs, dtype=np.uint8)
    n, L = s.shape
    out = np.zeros((n, n, 3), dtype=np.uint32)
    lib().orc_counts(s.tobytes(), n, L, type_, int(naive), int(full), out.reshape(-1))
    return out


def matrix(cnt: np.ndarray, L: int, type_: int, model: int, naive: bool = False,
           compat_wrap: bool = False, full: bool = False):
    """Post-processed float32 matrix and its maximum from counts."""
    n = cnt.shape[0]
    out = np.zeros((n, n), dtype=np.float32)
    fn = lib().orc_matrix_full if full else lib().orc_matrix
    mx = fn(np.ascontiguousarray(cnt, dtype=np.uint32).reshape(-1), n, L, type_, model,
            int(naive), int(compat_wrap), out.reshape(-1))
    return out, float(mx)


def raw_distances(cnt: np.ndarray, L: int, type_: int, model: int, naive: bool = False,
                  compat_wrap: bool = False, full: bool = False) -> np.ndarray:
    """Distances before the post-process (saturated pairs are -1) for j > i (every
    pair when ``full``); other entries zero."""
    n = cnt.shape[0]
    out = np.zeros((n, n), dtype=np.float32)
    lib().orc_raw_distances(np.ascontiguousarray(cnt, dtype=np.uint32).reshape(-1), n, L, type_,
                            model, int(naive), int(compat_wrap), int(full), out.reshape(-1))
    return out


def distance_matrix(seqs: np.ndarray, model: int, type_: int | None = None, naive: bool = False,
                    compat_wrap: bool = False):
    if type_ is None:
        type_ = detect_type(seqs)
    c = counts(seqs, type_, naive)
    return matrix(c, seqs.shape[1], type_, model, naive, compat_wrap)


# --- the reference itself -------------------------------------------------------

def ref_available() -> bool:
    return os.path.exists(REF_HARNESS)


def ref_counts(path: str, fmt: str = "fa", type_: str = "auto", fastdist: bool = True,
               full: bool = False):
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "c.bin")
        subprocess.run([REF_HARNESS, "counts", path, fmt, type_, str(int(fastdist)),
                        str(int(full)), out], check=True)
        raw = np.fromfile(out, dtype=np.int32, count=3)
        n, L, t = (int(x) for x in raw)
        c = np.fromfile(out, dtype=np.uint32, offset=12).reshape(n, n, 3)
    return c, L, t


def ref_matrix(path: str, model: str, fmt: str = "fa", type_: str = "auto",
               fastdist: bool = True, threads: int = 1, disk: bool = False,
               want_matrix: bool = True):
    """Runs the reference driver; returns (matrix or None, timing dict)."""
    with tempfile.TemporaryDirectory() as td:
        out = os.path.join(td, "m.bin") if want_matrix else "-"
        args = [REF_HARNESS, "matrix", path, fmt, type_, str(int(fastdist)), model,
                str(threads), out]
        if disk:
            args.append("disk")
        env = dict(os.environ, TMPDIR=td)
        p = subprocess.run(args, check=True, capture_output=True, text=True, env=env)
        info = json.loads(p.stdout.strip().splitlines()[-1])
        m = None
        if want_matrix:
            n = int(np.fromfile(out, dtype=np.int32, count=1)[0])
            m = np.fromfile(out, dtype=np.float32, offset=4).reshape(n, n)
    return m, info
