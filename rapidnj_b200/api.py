"""Python face of the C ABI: contexts, packed alignments, distance matrices.

Everything here forwards to librnjgpu.so; device buffers may be torch CUDA
tensors (passed by data pointer).  Host arrays are numpy.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from ._native import (RNJ_COMPAT_PROTEIN_WRAP, RNJ_DNA, RNJ_FASTDIST, RNJ_FULL_ROWS, RNJ_JC,
                      RNJ_KIMURA, RNJ_POPCOUNT, RNJ_PROTEIN, RNJ_UNKNOWN, check)

MODELS = {"jc": RNJ_JC, "kim": RNJ_KIMURA, RNJ_JC: RNJ_JC, RNJ_KIMURA: RNJ_KIMURA}
TYPES = {None: RNJ_UNKNOWN, "d": RNJ_DNA, "p": RNJ_PROTEIN, "dna": RNJ_DNA, "protein": RNJ_PROTEIN,
         RNJ_DNA: RNJ_DNA, RNJ_PROTEIN: RNJ_PROTEIN, RNJ_UNKNOWN: RNJ_UNKNOWN}


def flags_of(fastdist: bool = True, compat_wrap: bool = False, full_rows: bool = False,
             popcount: bool = False) -> int:
    return ((RNJ_FASTDIST if fastdist else 0) | (RNJ_COMPAT_PROTEIN_WRAP if compat_wrap else 0)
            | (RNJ_FULL_ROWS if full_rows else 0) | (RNJ_POPCOUNT if popcount else 0))


def detect_type(seq0: bytes) -> int:
    return N.lib().rnj_detect_type(seq0, len(seq0))


def version() -> str:
    return N.lib().rnj_version().decode()


class Alignment:
    """A packed alignment on the device (rnj_aln)."""

    def __init__(self, ctx: "Context", handle: int):
        self.ctx = ctx
        self.handle = ctypes.c_void_p(handle)
        n, L, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(N.lib().rnj_aln_info(self.handle, ctypes.byref(n), ctypes.byref(L), ctypes.byref(t)))
        self.n, self.L, self.type = n.value, L.value, t.value

    def close(self) -> None:
        # After its context is closed the native object is gone with it.
        if self.handle and self.ctx.handle:
            N.lib().rnj_aln_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Matrix:
    """A post-processed distance matrix on the device (rnj_mat)."""

    def __init__(self, ctx: "Context", handle: int):
        self.ctx = ctx
        self.handle = ctypes.c_void_p(handle)
        n = ctypes.c_int()
        check(N.lib().rnj_mat_info(self.handle, ctypes.byref(n), None))
        self.n = n.value

    @property
    def max(self) -> float:
        m = ctypes.c_float()
        check(N.lib().rnj_mat_info(self.handle, None, ctypes.byref(m)))
        return m.value

    def device_ptr(self):
        p, ld = ctypes.c_void_p(), ctypes.c_size_t()
        check(N.lib().rnj_mat_device_ptr(self.handle, ctypes.byref(p), ctypes.byref(ld)))
        return p.value, ld.value

    def copy_rows(self, rows, row0: int = 0, threads: int = 0) -> None:
        """Copies len(rows) rows starting at row0 into host float32 arrays."""
        ptrs = (ctypes.c_void_p * len(rows))(*[r.ctypes.data for r in rows])
        check(N.lib().rnj_mat_copy_rows(self.ctx.handle, self.handle, row0, len(rows), ptrs, threads))

    def to_numpy(self, threads: int = 0) -> np.ndarray:
        out = np.empty((self.n, self.n), dtype=np.float32)
        self.copy_rows([out[i] for i in range(self.n)], 0, threads)
        return out

    def close(self) -> None:
        if self.handle and self.ctx.handle:
            N.lib().rnj_mat_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One device, one CUDA stream (rnj_ctx)."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        check(N.lib().rnj_ctx_create(device, ctypes.byref(h)))
        self.handle = h
        self.device = device

    @property
    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(N.lib().rnj_ctx_stream(self.handle, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self) -> None:
        check(N.lib().rnj_ctx_synchronize(self.handle))

    def set_profiling(self, on: bool = True) -> None:
        check(N.lib().rnj_ctx_set_profiling(self.handle, int(on)))

    def stage_times(self):
        """(pack_ms, count_ms, fixup_ms) of the last call, profiling on."""
        ms = (ctypes.c_float * 3)()
        check(N.lib().rnj_ctx_stage_times(self.handle, ms))
        return tuple(ms)

    def probe_int_peaks(self):
        """(POPC ops/s, LOP3 ops/s) measured on this device."""
        a, b = ctypes.c_double(), ctypes.c_double()
        check(N.lib().rnj_probe_int_peaks(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def probe_tc_peak(self) -> float:
        """FP4 tensor-pipe flop/s measured on this device (back-to-back 128 x 128 x 64
        kind::mxf4 MMAs on every SM)."""
        x = ctypes.c_double()
        check(N.lib().rnj_probe_tc_peak(self.handle, ctypes.byref(x)))
        return x.value

    def check_quotient16(self) -> int:
        """Mismatches of the fused epilogue's quotients, checked on the device over
        their whole domains: the float quotients num / n (0 <= num <= n < 2^16)
        and JC's double p / b (every float p in [0, 1], b = 3/4 and 19/20).  0 on
        a sound build."""
        x = ctypes.c_ulonglong()
        check(N.lib().rnj_check_quotient16(self.handle, ctypes.byref(x)))
        return x.value

    # --- alignments
    def alignment(self, seqs, type_=None, fastdist: bool = True, compat_wrap: bool = False,
                  full_rows: bool = False, popcount: bool = False) -> Alignment:
        """Packs an alignment from a host (n, L) uint8 array or a CUDA uint8 tensor."""
        flags = flags_of(fastdist, compat_wrap, full_rows, popcount)
        t = TYPES[type_]
        h = ctypes.c_void_p()
        if hasattr(seqs, "is_cuda") and seqs.is_cuda:
            n, L = seqs.shape
            ld = seqs.stride(0)
            check(N.lib().rnj_aln_from_device(self.handle, ctypes.c_void_p(seqs.data_ptr()), n, L,
                                              ld, t, flags, ctypes.byref(h)))
        else:
            a = np.ascontiguousarray(seqs, dtype=np.uint8)
            n, L = a.shape
            check(N.lib().rnj_aln_from_host_buffer(self.handle, a.ctypes.data, n, L, L, t, flags,
                                                   ctypes.byref(h)))
        return Alignment(self, h.value)

    def alignment_from_rows(self, rows, type_=None, fastdist=True, compat_wrap=False,
                            full_rows=False) -> Alignment:
        """Packs from a list of equal-length bytes objects (row pointers)."""
        n = len(rows)
        L = len(rows[0]) if n else 0
        arr = (ctypes.c_char_p * n)(*rows)
        h = ctypes.c_void_p()
        check(N.lib().rnj_aln_from_host(self.handle, arr, n, L, TYPES[type_],
                                        flags_of(fastdist, compat_wrap, full_rows), ctypes.byref(h)))
        return Alignment(self, h.value)

    def alignment_from_bitstrings(self, bit_strings, gap_filters, L: int, type_: int,
                                  flags: int = RNJ_FASTDIST) -> Alignment:
        """From the reference loader's packed arrays (lists of uint32 numpy arrays of
        bitStringsCount * 4 words each)."""
        n = len(bit_strings)
        count = bit_strings[0].size // 4 if n else 0
        bs = (ctypes.c_void_p * n)(*[b.ctypes.data for b in bit_strings])
        gf = (ctypes.c_void_p * n)(*[g.ctypes.data for g in gap_filters]) if gap_filters else None
        h = ctypes.c_void_p()
        check(N.lib().rnj_aln_from_bitstrings(self.handle, bs, gf, n, L, count, type_, flags,
                                              ctypes.byref(h)))
        return Alignment(self, h.value)

    # --- distances
    def distance(self, aln: Alignment, model="kim") -> Matrix:
        h = ctypes.c_void_p()
        check(N.lib().rnj_distance(self.handle, aln.handle, MODELS[model], ctypes.byref(h)))
        return Matrix(self, h.value)

    def distance_into(self, aln: Alignment, model, out, want_max: bool = False):
        """Into a CUDA float32 tensor of shape (n, >= n).  Returns the max when asked
        (synchronising), else None."""
        m = ctypes.c_float()
        check(N.lib().rnj_distance_into(self.handle, aln.handle, MODELS[model],
                                        ctypes.c_void_p(out.data_ptr()), out.stride(0),
                                        ctypes.byref(m) if want_max else None))
        return m.value if want_max else None

    def distance_f64(self, aln: Alignment, model, out=None):
        """rnj_distance_f64: the matrix in double precision (each pair's value is
        the reference's double before its float cast) into a CUDA float64 tensor
        (n, >= n), allocated when out is None.  Returns (tensor, max)."""
        import torch
        if out is None:
            out = torch.empty((aln.n, aln.n), dtype=torch.float64, device=f"cuda:{self.device}")
        m = ctypes.c_double()
        check(N.lib().rnj_distance_f64(self.handle, aln.handle, MODELS[model],
                                       ctypes.c_void_p(out.data_ptr()), out.stride(0),
                                       ctypes.byref(m)))
        return out, m.value

    def distance_rows(self, aln: Alignment, model, on_rows, band_rows: int = 0):
        """The matrix in bands of full rows (rnj_distance_rows), for matrices larger
        than device memory: on_rows(row0, rows) receives each band as a float32
        array view (valid during the call; copy what you keep), rows as the
        reference's disk-matrix drivers write them (diagonal 0, saturated pairs -1).
        Returns (max distance, whether a pair saturated)."""
        err = []

        def cb(_user, row0, nrows, ptr, ld):
            try:
                arr = np.ctypeslib.as_array(ptr, shape=(nrows, ld))
                on_rows(row0, arr[:, :aln.n])
                return 0
            except Exception as e:  # noqa: BLE001 -- reported after the call
                err.append(e)
                return 1

        fn = N.ROWS_FN(cb)
        mx, sat = ctypes.c_float(), ctypes.c_int()
        st = N.lib().rnj_distance_rows(self.handle, aln.handle, MODELS[model], band_rows,
                                       ctypes.cast(fn, ctypes.c_void_p), None, ctypes.byref(mx),
                                       ctypes.byref(sat))
        if err:
            raise err[0]
        check(st)
        return mx.value, bool(sat.value)

    def memory(self):
        """(free, total) bytes of the context's device."""
        f, t = ctypes.c_size_t(), ctypes.c_size_t()
        check(N.lib().rnj_ctx_memory(self.handle, ctypes.byref(f), ctypes.byref(t)))
        return f.value, t.value

    def counts_into(self, aln: Alignment, out) -> None:
        """Raw counts into a CUDA int32/uint32 tensor of n*n*3 elements."""
        check(N.lib().rnj_counts_into(self.handle, aln.handle, ctypes.c_void_p(out.data_ptr())))

    def distance_matrix_host(self, seqs: np.ndarray, model="kim", type_=None, fastdist=True,
                             compat_wrap=False, full_rows=False, popcount=False, out=None,
                             band_tiles=None):
        """Host bytes in, host n x n float32 matrix out (``out``, C-contiguous, may be
        page-locked memory, which the library then fills by direct DMA).

        ``band_tiles`` (rnj_distance_matrix_host_ex): None or 0 = the library's
        choice, > 0 = band height in 128-row tiles of the streamed form, < 0 =
        not streamed."""
        a = np.ascontiguousarray(seqs, dtype=np.uint8)
        n, L = a.shape
        if out is None:
            out = np.empty((n, n), dtype=np.float32)
        assert out.dtype == np.float32 and out.shape == (n, n) and out.flags.c_contiguous
        m = ctypes.c_float()
        flags = flags_of(fastdist, compat_wrap, full_rows, popcount)
        if band_tiles is None:
            check(N.lib().rnj_distance_matrix_host(self.handle, a.ctypes.data, n, L, L,
                                                   TYPES[type_], MODELS[model], flags,
                                                   out.ctypes.data, ctypes.byref(m)))
        else:
            check(N.lib().rnj_distance_matrix_host_ex(self.handle, a.ctypes.data, n, L, L,
                                                      TYPES[type_], MODELS[model], flags,
                                                      int(band_tiles), out.ctypes.data,
                                                      ctypes.byref(m)))
        return out, m.value

    def bootstrap(self, d_chars, columns: np.ndarray, type_, model="kim", fastdist: bool = True,
                  outs=None):
        """rnj_bootstrap: replicate r of the device alignment d_chars (a CUDA uint8
        tensor, n x L) takes column columns[r, k] as its column k.  Returns the
        list of R device matrices (n x n float32 tensors) and their maxima."""
        import torch
        n, L = d_chars.shape
        cols = np.ascontiguousarray(columns, dtype=np.int32)
        R = cols.shape[0]
        assert cols.shape == (R, L)
        if outs is None:
            outs = [torch.empty((n, n), dtype=torch.float32, device=d_chars.device)
                    for _ in range(R)]
        ptrs = (ctypes.c_void_p * max(R, 1))(*[o.data_ptr() for o in outs])
        mx = np.zeros(max(R, 1), dtype=np.float32)
        check(N.lib().rnj_bootstrap(self.handle, ctypes.c_void_p(d_chars.data_ptr()), n, L,
                                    d_chars.stride(0), TYPES[type_], MODELS[model],
                                    flags_of(fastdist), R, cols.ctypes.data, ptrs, n,
                                    mx.ctypes.data))
        return outs, mx[:R]

    def read_alignment_device(self, path: str, fmt: str | None = None):
        """rnj_msa_read_device: the file parsed on this context's device.  Returns
        (names, chars: CUDA uint8 tensor (n, L), detected type), the same names and
        bytes as read_alignment."""
        import torch
        h = ctypes.c_void_p()
        check(N.lib().rnj_msa_read_device(self.handle, path.encode(),
                                          fmt.encode() if fmt else None, ctypes.byref(h)))
        try:
            names, n, L, t = _msa_header(h)
            if n * L == 0:
                return names, torch.zeros((n, L), dtype=torch.uint8, device=f"cuda:{self.device}"), t
            p, ld = ctypes.c_void_p(), ctypes.c_size_t()
            check(N.lib().rnj_msa_device_chars(h, ctypes.byref(p), ctypes.byref(ld)))

            class _View:  # the library's device bytes, copied before the handle goes
                __cuda_array_interface__ = {"shape": (n, L), "typestr": "|u1",
                                            "data": (p.value, False), "version": 3,
                                            "strides": (ld.value, 1)}
            with torch.cuda.device(self.device):
                chars = torch.as_tensor(_View(), device=f"cuda:{self.device}").clone()
            return names, chars, t
        finally:
            N.lib().rnj_msa_destroy(h)

    def nj_init(self, d_matrix, cap: int = 0, sorted_rows: bool = True, sorted_out=None):
        """rnj_nj_init: rapidNJ's set-up over the device distance matrix d_matrix (a
        CUDA float32 tensor, n x n, row stride >= n).  Returns a dict of host arrays
        (separation_sums, separations, max_row_separations, max_separation,
        possible_redundant, index_to_id, redundant_to_master, redundant_count,
        row_lengths) and, when sorted_rows, ``sorted``: a device int32 tensor
        (n, ld, 2) of (id, distance bits) pairs (``sorted_distances`` views the
        distances as float32).  cap > 0 keeps rapidNJMem's first cap entries."""
        import torch
        n = d_matrix.shape[0]
        assert d_matrix.dtype == torch.float32 and d_matrix.shape == (n, n)
        assert d_matrix.stride(1) == 1
        res = {"separation_sums": np.zeros(n, np.float32), "separations": np.zeros(n, np.float32),
               "max_row_separations": np.zeros(n, np.float32),
               "max_separation": np.zeros(1, np.float32),
               "possible_redundant": np.zeros(n, np.int16),
               "index_to_id": np.zeros(n, np.int32), "redundant_to_master": np.zeros(n, np.int32),
               "redundant_count": np.zeros(n, np.int32), "row_lengths": np.zeros(n, np.int32)}
        d = N.NjData()
        for k, a in res.items():
            setattr(d, k, a.ctypes.data)
        d.sorted_cap = int(cap)
        if sorted_rows:
            width = max(1, min(cap, n - 1) if cap > 0 else n - 1)
            if sorted_out is None:
                sorted_out = torch.zeros((n, width, 2), dtype=torch.int32, device=d_matrix.device)
            assert sorted_out.dtype == torch.int32 and sorted_out.shape[0] == n
            assert sorted_out.shape[2] == 2 and sorted_out.is_contiguous()
            d.sorted = sorted_out.data_ptr()
            d.sorted_ld = sorted_out.shape[1]
        check(N.lib().rnj_nj_init(self.handle, ctypes.c_void_p(d_matrix.data_ptr()), n,
                                  d_matrix.stride(0), ctypes.byref(d)))
        res["max_separation"] = res["max_separation"][0]
        if sorted_rows:
            res["sorted"] = sorted_out
            res["sorted_distances"] = sorted_out[..., 1].view(torch.float32)
        return res

    def tune(self, n: int, L: int, type_="dna", fastdist: bool = True,
             popcount: bool = False) -> "TuneParams":
        """rnj_tune: time the candidate launch choices of the bucket of (n, L) on a
        seeded synthetic n x L alignment and keep the fastest for later calls
        (popcount: only the bit-plane kernels' choices)."""
        p = TuneParams()
        check(N.lib().rnj_tune(self.handle, n, L, TYPES[type_],
                               flags_of(fastdist, popcount=popcount), ctypes.byref(p)))
        return p

    def close(self) -> None:
        if self.handle:
            N.lib().rnj_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many alignments in one persistent pass (rnj_batch): a device work list of
    all their tiles, consumed by graph-captured persistent kernels."""

    def __init__(self, ctx: Context, max_alignments: int = 1024, max_tiles: int = 1 << 16):
        h = ctypes.c_void_p()
        check(N.lib().rnj_batch_create(ctx.handle, max_alignments, max_tiles, ctypes.byref(h)))
        self.ctx = ctx
        self.handle = h
        self._keep = []

    def add(self, aln: Alignment, model="kim", out=None) -> int:
        """Adds a packed alignment; out (CUDA float32 tensor n x >= n) or None."""
        slot = ctypes.c_int()
        ptr = ctypes.c_void_p(out.data_ptr()) if out is not None else None
        ld = out.stride(0) if out is not None else 0
        check(N.lib().rnj_batch_add(self.handle, aln.handle, MODELS[model], ptr, ld,
                                    ctypes.byref(slot)))
        self._keep.append(aln)
        return slot.value

    def add_many(self, seqs_dev, types, models, outs=None, fastdist=True, popcount=False):
        """Packs and adds CUDA uint8 tensors (n x L views) in one call; returns slots."""
        k = len(seqs_dev)
        ptrs = (ctypes.c_void_p * k)(*[s.data_ptr() for s in seqs_dev])
        ns = (ctypes.c_int * k)(*[s.shape[0] for s in seqs_dev])
        Ls = (ctypes.c_int * k)(*[s.shape[1] for s in seqs_dev])
        lds = (ctypes.c_size_t * k)(*[s.stride(0) for s in seqs_dev])
        ts = (ctypes.c_int * k)(*[TYPES[t] for t in types])
        ms = (ctypes.c_int * k)(*[MODELS[m] for m in models])
        outp = (ctypes.c_void_p * k)(*[o.data_ptr() for o in outs]) if outs is not None else None
        ldo = (ctypes.c_size_t * k)(*[o.stride(0) for o in outs]) if outs is not None else None
        slots = (ctypes.c_int * k)()
        check(N.lib().rnj_batch_add_many(self.handle, k, ptrs, ns, Ls, lds, ts, ms,
                                         flags_of(fastdist, False, False, popcount), outp, ldo,
                                         slots))
        return list(slots)

    def run(self) -> None:
        check(N.lib().rnj_batch_run(self.handle))

    def synchronize(self) -> None:
        check(N.lib().rnj_batch_synchronize(self.handle))

    def max(self, slot: int) -> float:
        m = ctypes.c_float()
        check(N.lib().rnj_batch_output(self.handle, slot, None, None, ctypes.byref(m)))
        return m.value

    def take(self, slot: int) -> Matrix:
        h = ctypes.c_void_p()
        check(N.lib().rnj_batch_take(self.handle, slot, ctypes.byref(h)))
        return Matrix(self.ctx, h.value)

    def size(self):
        a, t = ctypes.c_int(), ctypes.c_longlong()
        check(N.lib().rnj_batch_size(self.handle, ctypes.byref(a), ctypes.byref(t)))
        return a.value, t.value

    def tuning(self):
        """(ring depth, alignments with a tuned entry) of the last run."""
        d, t = ctypes.c_int(), ctypes.c_int()
        check(N.lib().rnj_batch_tuning(self.handle, ctypes.byref(d), ctypes.byref(t)))
        return d.value, t.value

    def clear(self) -> None:
        check(N.lib().rnj_batch_clear(self.handle))
        self._keep = []

    def close(self) -> None:
        if self.handle and self.ctx.handle:
            N.lib().rnj_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TuneParams(ctypes.Structure):
    """rnj_tune_params: the launch choices of one bucket (alphabet, rules,
    floor(log2 n), floor(log2 L)); zero fields mean the library default."""
    _fields_ = [("dna_kernel", ctypes.c_int), ("ksplit", ctypes.c_int),
                ("tile_band", ctypes.c_int), ("transform_ctas", ctypes.c_int),
                ("stream_band", ctypes.c_int), ("tc_epilogue", ctypes.c_int),
                ("tc_stages", ctypes.c_int), ("pop_stages", ctypes.c_int),
                ("ms", ctypes.c_float)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def tune_get(n: int, L: int, type_="dna", fastdist: bool = True):
    """The stored entry of the bucket of (n, L), or None."""
    p = TuneParams()
    rc = N.lib().rnj_tune_get(n, L, TYPES[type_], flags_of(fastdist), ctypes.byref(p))
    if rc == 9:  # RNJ_ERR_NOTREADY: no entry for this bucket
        return None
    check(rc)
    return p


def tune_set(n: int, L: int, type_="dna", fastdist: bool = True, **fields) -> None:
    p = TuneParams(**fields)
    check(N.lib().rnj_tune_set(n, L, TYPES[type_], flags_of(fastdist), ctypes.byref(p)))


def tune_clear() -> None:
    check(N.lib().rnj_tune_clear())


def tune_save(path: str) -> None:
    check(N.lib().rnj_tune_save(path.encode()))


def tune_load(path: str) -> None:
    check(N.lib().rnj_tune_load(path.encode()))


def shard_tiles(n: int, shard: int, nshards: int, full_rows: bool = False):
    """(tile0, tile1, ntiles): the contiguous tile range of one shard (host only)."""
    t0, t1, nt = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    check(N.lib().rnj_shard_tiles(n, int(full_rows), shard, nshards, ctypes.byref(t0),
                                  ctypes.byref(t1), ctypes.byref(nt)))
    return t0.value, t1.value, nt.value


def tile_coords(n: int, tile: int, full_rows: bool = False):
    """(tile_row, tile_col) of a linear tile index (host only)."""
    r, c = ctypes.c_int(), ctypes.c_int()
    check(N.lib().rnj_tile_coords(n, int(full_rows), tile, ctypes.byref(r), ctypes.byref(c)))
    return r.value, c.value


class Shard:
    """One GPU's share of one alignment's tiles (rnj_shard): run() gives the
    local maximum, finish(global_max) applies the saturation cap."""

    def __init__(self, ctx: Context, aln: Alignment, model, shard: int, nshards: int, out=None):
        h = ctypes.c_void_p()
        ptr = ctypes.c_void_p(out.data_ptr()) if out is not None else None
        ld = out.stride(0) if out is not None else 0
        check(N.lib().rnj_shard_create(ctx.handle, aln.handle, MODELS[model], shard, nshards, ptr,
                                       ld, ctypes.byref(h)))
        self.ctx, self.aln, self.handle = ctx, aln, h
        self.n = aln.n

    def run(self) -> float:
        m = ctypes.c_float()
        check(N.lib().rnj_shard_run(self.handle, ctypes.byref(m)))
        return m.value

    def finish(self, global_max: float) -> None:
        check(N.lib().rnj_shard_finish(self.handle, ctypes.c_float(global_max)))

    def output(self):
        p, ld = ctypes.c_void_p(), ctypes.c_size_t()
        check(N.lib().rnj_shard_output(self.handle, ctypes.byref(p), ctypes.byref(ld)))
        return p.value, ld.value

    def copy_tiles(self, host: np.ndarray) -> int:
        """Copies this shard's tiles into a float32 (n, >= n) C-contiguous host array."""
        assert host.dtype == np.float32 and host.flags.c_contiguous and host.shape[0] == self.n
        nbytes = ctypes.c_size_t()
        check(N.lib().rnj_shard_copy_tiles(self.handle, host.ctypes.data, host.shape[1],
                                           ctypes.byref(nbytes)))
        return nbytes.value

    def close(self) -> None:
        if self.handle and self.ctx.handle:
            N.lib().rnj_shard_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching distance server (rnj_server) with its own device context."""

    def __init__(self, device: int = 0, memory_budget: int = 0, max_batch: int = 256):
        h = ctypes.c_void_p()
        check(N.lib().rnj_server_create(device, memory_budget, max_batch, ctypes.byref(h)))
        self.handle = h

    def submit(self, seqs: np.ndarray, model="kim", type_=None, fastdist=True,
               popcount=False) -> int:
        a = np.ascontiguousarray(seqs, dtype=np.uint8)
        n, L = a.shape
        rid = ctypes.c_uint64()
        check(N.lib().rnj_server_submit(self.handle, a.ctypes.data, n, L, L, TYPES[type_],
                                        MODELS[model], flags_of(fastdist, False, False, popcount),
                                        ctypes.byref(rid)))
        return rid.value

    def state(self, rid: int) -> int:
        s = ctypes.c_int()
        check(N.lib().rnj_server_poll(self.handle, rid, ctypes.byref(s)))
        return s.value

    def wait(self, rid: int, timeout_ms: int = 60000) -> None:
        check(N.lib().rnj_server_wait(self.handle, rid, timeout_ms))

    def result(self, ctx: Context, rid: int):
        """(Matrix on the device, latency in ms); the matrix belongs to the caller."""
        h = ctypes.c_void_p()
        lat = ctypes.c_double()
        check(N.lib().rnj_server_result(self.handle, rid, ctx.handle, ctypes.byref(h),
                                        ctypes.byref(lat)))
        m = Matrix(ctx, h.value)
        return m, lat.value

    def stats(self):
        c, w, s, b = ctypes.c_uint64(), ctypes.c_double(), ctypes.c_double(), ctypes.c_size_t()
        check(N.lib().rnj_server_stats(self.handle, ctypes.byref(c), ctypes.byref(w),
                                       ctypes.byref(s), ctypes.byref(b)))
        return {"completed": c.value, "pair_columns": w.value, "seconds": s.value,
                "bytes_in_use": b.value}

    def close(self) -> None:
        if self.handle:
            N.lib().rnj_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --- alignment files (host only) -------------------------------------------------

def _msa_header(h):
    """(names, n, L, detected type) of an rnj_msa handle."""
    n, L, t = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(N.lib().rnj_msa_info(h, ctypes.byref(n), ctypes.byref(L), ctypes.byref(t)))
    names = []
    k = 0
    while True:
        nm = N.lib().rnj_msa_name(h, k)
        if nm is None:
            break
        names.append(nm.decode("latin-1"))
        k += 1
    return names, n.value, L.value, t.value


def read_alignment(path: str, fmt: str | None = None):
    """(names, chars (n, L) uint8, detected type) with the reference loaders' rules."""
    h = ctypes.c_void_p()
    check(N.lib().rnj_msa_read(path.encode(), fmt.encode() if fmt else None, ctypes.byref(h)))
    try:
        names, n, L, t = _msa_header(h)
        ptr = N.lib().rnj_msa_chars(h)
        size = n * L
        chars = np.ctypeslib.as_array((ctypes.c_uint8 * size).from_address(ptr)) \
            .reshape(n, L).copy() if size else np.zeros((n, L), np.uint8)
        return names, chars, t
    finally:
        N.lib().rnj_msa_destroy(h)


def write_matrix_text_device(ctx: "Context", path: str | None, names, d_matrix) -> None:
    """rnj_write_matrix_text_device: the "-o m" text of a CUDA float32 (n, n) tensor
    (row stride >= n), formatted on the device; byte-identical to
    write_matrix_text."""
    n = d_matrix.shape[0]
    assert d_matrix.shape == (n, n) and d_matrix.stride(1) == 1
    nm = (ctypes.c_char_p * max(n, 1))(*[x.encode("latin-1") for x in names[:n]])
    check(N.lib().rnj_write_matrix_text_device(ctx.handle, path.encode() if path else None, nm,
                                               ctypes.c_void_p(d_matrix.data_ptr()),
                                               d_matrix.stride(0), n))


def write_matrix_text(path: str | None, names, matrix: np.ndarray, threads: int = 0) -> None:
    m = np.ascontiguousarray(matrix, dtype=np.float32)
    n = m.shape[0]
    nm = (ctypes.c_char_p * n)(*[x.encode("latin-1") for x in names[:n]])
    rows = (ctypes.c_void_p * n)(*[m[i].ctypes.data for i in range(n)])
    check(N.lib().rnj_write_matrix_text(path.encode() if path else None, nm, rows, n, threads))
