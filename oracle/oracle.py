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


def reference_tree() -> str | None:
    """The rapidNJ source tree the harnesses are compiled from: $RNJ_REFERENCE, else a
    ``reference`` folder beside this repository; None when neither exists."""
    env = os.environ.get("RNJ_REFERENCE")
    if env:
        return env if os.path.isdir(env) else None
    beside = os.path.abspath(os.path.join(HERE, "..", "..", "reference"))
    return beside if os.path.isdir(os.path.join(beside, "src")) else None


def build() -> None:
    """Compile liborc.so (and the reference harness when the reference tree is
    present)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = reference_tree()
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + ref], check=True)
        if os.path.exists(os.path.join(HERE, "..", "rapidnj_b200", "librnjgpu.so")):
            subprocess.run(["make", "-s", "-C", HERE, "dropin", "REF=" + ref], check=True)


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
        L.orc_counts_rows.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.c_void_p]
        L.orc_counts_rows.restype = None
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
        f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        L.orc_matrix_d.argtypes = [u32p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int, f64p]
        L.orc_matrix_d.restype = ctypes.c_double
        for name in ("orc_jc_d", "orc_k2p_d", "orc_kimura_protein_d"):
            getattr(L, name).restype = ctypes.c_double
        L.orc_jc_d.argtypes = [ctypes.c_uint64] * 3 + [ctypes.c_int]
        L.orc_k2p_d.argtypes = [ctypes.c_uint64] * 3
        L.orc_kimura_protein_d.argtypes = [ctypes.c_uint64] * 2
        _lib = L
    return _lib


def detect_type(seqs: np.ndarray) -> int:
    row = np.ascontiguousarray(seqs[0], dtype=np.uint8)
    return lib().orc_detect_type(row.tobytes(), row.size)


def counts(seqs: np.ndarray, type_: int, naive: bool = False, full: bool = False,
           threads: int = 1) -> np.ndarray:
    """(n, n, 3) uint32: {ts, tv, valid} (DNA) or {mismatch, 0, valid} (protein)
    for j > i (every pair when ``full``).  ``threads`` > 1 splits the rows into
    ranges of equal pair count, one host thread each (the C calls release the GIL)."""
    s = np.ascontiguousarray(seqs, dtype=np.uint8)
    n, L = s.shape
    out = np.zeros((n, n, 3), dtype=np.uint32)
    if threads <= 1 or n < 4:
        lib().orc_counts(s.tobytes(), n, L, type_, int(naive), int(full), out.reshape(-1))
        return out
    from concurrent.futures import ThreadPoolExecutor
    raw = s.tobytes()
    # row i holds n - 1 - i pairs (n with ``full``): cut at equal cumulative work
    work = np.full(n, n, np.float64) if full else np.arange(n - 1, -1, -1, dtype=np.float64)
    cum = np.concatenate([[0.0], np.cumsum(work)])
    cuts = [int(np.searchsorted(cum, cum[-1] * k / threads)) for k in range(threads + 1)]
    cuts[0], cuts[-1] = 0, n
    ptr = out.ctypes.data
    with ThreadPoolExecutor(threads) as ex:
        list(ex.map(lambda k: lib().orc_counts_rows(raw, n, L, type_, int(naive), int(full),
                                                    cuts[k], cuts[k + 1], ptr)
                    if cuts[k + 1] > cuts[k] else None, range(threads)))
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


def matrix_f64(cnt: np.ndarray, L: int, type_: int, model: int, naive: bool = False,
               compat_wrap: bool = False, full: bool = False):
    """The double matrix (each pair's value before the reference's float cast,
    post-processed in double) and its maximum from counts (orc_matrix_d)."""
    n = cnt.shape[0]
    out = np.zeros((n, n), dtype=np.float64)
    mx = lib().orc_matrix_d(np.ascontiguousarray(cnt, dtype=np.uint32).reshape(-1), n, L, type_,
                            model, int(naive), int(compat_wrap), int(full), out.reshape(-1))
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


# --- neighbour-joining set-up ---------------------------------------------------

FLT_MIN = np.float32(1.17549435e-38)


def nj_init(m: np.ndarray, cap: int = 0) -> dict:
    """Restatement of the reference's NJ initialisation over an n x n float32
    distance matrix (rapidNJ::initialize, rapidNJ.cpp:94-141; rapidNJMem::initialize,
    rapidNJMem.cpp:92-135 when cap > 0 is its sortedMatrixSize), for small n.

    * separation sums: float32 sum of row i in column order (rapidNJ.cpp:107-110),
      separations = sum / (n - 2) in float32 (:111), maxRowSeparations[i] = the
      largest separation of rows before i, FLT_MIN first (:102,113-118);
    * redundant rows: i from n-1 down, skipping rows already marked; for j < i with
      m[i][j] == 0 and rows i and j equal everywhere (float ==), j is marked
      (indexToId -1), mapped to i and pushed to the front of i's list
      (:121-131, handleRedundancy :156-167);
    * sorted rows: for each unmarked row i the unmarked j < i as (id, m[i][j]),
      sorted by distance (:134-154), the first `cap` kept for rapidNJMem
      (rapidNJMem.cpp:138-153).  std::sort leaves the order of equal distances
      unspecified; this restatement keeps them in id order.
    * possible_redundant: the row has a zero off the diagonal
      (rdDataInitialiser::processRow, rdDataInitialiser.cpp:174-189).
    """
    m = np.ascontiguousarray(m, dtype=np.float32)
    n = m.shape[0]
    sums = np.cumsum(m, axis=1, dtype=np.float32)[:, -1] if n else np.zeros(0, np.float32)
    with np.errstate(divide="ignore", invalid="ignore"):
        seps = (sums / np.float32(n - 2)).astype(np.float32)
    maxrow = np.empty(n, np.float32)
    mx = FLT_MIN
    for i in range(n):
        maxrow[i] = mx
        if seps[i] > mx:
            mx = seps[i]
    index_to_id = np.arange(n, dtype=np.int32)
    master = np.arange(n, dtype=np.int32)
    count = np.ones(n, dtype=np.int32)
    lists = [[] for _ in range(n)]
    for i in range(n - 1, -1, -1):
        if index_to_id[i] == -1:
            continue
        for j in np.nonzero(m[i, :i] == 0)[0]:
            if np.all(m[i] == m[j]):
                index_to_id[j] = -1
                master[j] = i
                lists[i].insert(0, int(j))
                count[i] += 1
    keep = index_to_id != -1
    lengths = np.zeros(n, dtype=np.int32)
    rows = []
    for i in range(n):
        if not keep[i]:
            rows.append(None)
            continue
        ids = np.nonzero(keep[:i])[0].astype(np.uint32)
        d = m[i, ids]
        order = np.argsort(d, kind="stable")
        k = len(ids) if cap <= 0 else min(len(ids), cap)
        lengths[i] = k
        rows.append((ids[order][:k], d[order][:k]))
    zero = (m == 0)
    np.fill_diagonal(zero, False)
    return {"sums": sums, "separations": seps, "max_row_separations": maxrow,
            "max_separation": np.float32(mx), "index_to_id": index_to_id,
            "redundant_to_master": master, "redundant_count": count, "lists": lists,
            "row_lengths": lengths, "rows": rows,
            "possible_redundant": zero.any(axis=1).astype(np.int16)}


def ref_nj_init(m: np.ndarray, cap: int = 0, reps: int = 1, want: bool = True):
    """The reference's own initialize() through _ref/nj_harness; returns the same
    dictionary as nj_init (without possible_redundant) and the timing line."""
    m = np.ascontiguousarray(m, dtype=np.float32)
    n = m.shape[0]
    with tempfile.TemporaryDirectory() as td:
        src = os.path.join(td, "m.bin")
        out = os.path.join(td, "o.bin") if want else "-"
        with open(src, "wb") as f:
            np.array([n, cap], dtype=np.int32).tofile(f)
            m.tofile(f)
        p = subprocess.run([os.path.join(REF_DIR, "nj_harness"), src, out, str(reps)],
                           check=True, capture_output=True, text=True)
        info = json.loads(p.stdout.strip().splitlines()[-1])
        if not want:
            return None, info
        raw = open(out, "rb").read()
    pos = 4
    def take(dt, k):
        nonlocal pos
        a = np.frombuffer(raw, dtype=dt, count=k, offset=pos).copy()
        pos += a.nbytes
        return a
    res = {"sums": take(np.float32, n), "separations": take(np.float32, n),
           "max_row_separations": take(np.float32, n),
           "max_separation": take(np.float32, 1)[0], "index_to_id": take(np.int32, n),
           "redundant_to_master": take(np.int32, n), "redundant_count": take(np.int32, n),
           "row_lengths": take(np.int32, n)}
    lists = []
    for _ in range(n):
        k = int(take(np.int32, 1)[0])
        lists.append([int(x) for x in take(np.int32, k)])
    res["lists"] = lists
    rows = []
    for i in range(n):
        k = int(res["row_lengths"][i])
        if res["index_to_id"][i] == -1:
            rows.append(None)
            continue
        pairs = take(np.uint32, 2 * k).reshape(k, 2)
        rows.append((pairs[:, 0].copy(), pairs[:, 1].view(np.float32).copy()))
    res["rows"] = rows
    return res, info
