"""rnj_distance_noalloc: distances for callers that cannot allocate device memory.

Who needs it: a process that owns the GPU through its own fixed memory pool (a
server that reserves device memory up front and forbids outside allocations),
or code that must not call cudaMalloc because it synchronises the device.  The
entry point takes the caller's device input, output and stream, and keeps its
intermediate buffers in one 16 MiB array built into the library.

The test calls it through the C ABI twice in a row and compares each result
with rnj_distance_into, the entry point that allocates; the two calls differ in
data so that state left by the first (the running maximum, the saturation
flags) would show in the second.  It lives in its own file, collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def ulp_diff(a, b):
    a = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return np.abs(a - b)


def noalloc(seqs_dev, typ, model, flags, out, stream=None):
    from rapidnj_b200 import _native
    n, L = seqs_dev.shape
    m = ctypes.c_float()
    st = _native.lib().rnj_distance_noalloc(
        ctypes.c_void_p(seqs_dev.data_ptr()), n, L, seqs_dev.stride(0), typ, model, flags,
        ctypes.c_void_p(out.data_ptr()), out.stride(0),
        ctypes.c_void_p(stream.cuda_stream if stream is not None else 0), ctypes.byref(m))
    return st, m.value


def existing(seqs_dev, typ, model, flags):
    from rapidnj_b200 import api
    ctx = api.Context(0)
    try:
        aln = ctx.alignment(seqs_dev, typ, fastdist=bool(flags & 1))
        n = seqs_dev.shape[0]
        out = torch.empty((n, n), dtype=torch.float32, device="cuda")
        mx = ctx.distance_into(aln, model, out, want_max=True)
        aln.close()
        return out.cpu().numpy(), mx
    finally:
        ctx.close()


def test_noalloc_matches_allocating_entry_on_two_calls():
    from rapidnj_b200 import synth
    from rapidnj_b200._native import RNJ_DNA, RNJ_FASTDIST, RNJ_KIMURA, RNJ_JC, RNJ_PROTEIN
    rng = np.random.default_rng(0)
    # call 1: many saturated pairs (unrelated short sequences), JC
    a = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (300, 48))]
    # call 2: tree-evolved, no saturation, Kimura-2P, with an odd row stride
    b = synth.tree_dna(700, 3000, seed=2, mean_branch=0.05)
    calls = [(a, RNJ_DNA, RNJ_JC), (b, RNJ_DNA, RNJ_KIMURA)]
    stream = torch.cuda.Stream()
    for k, (seqs, typ, model) in enumerate(calls):
        n, L = seqs.shape
        dev = torch.zeros((n, L + 5), dtype=torch.uint8, device="cuda")
        dev[:, :L] = torch.from_numpy(seqs).cuda()
        dev = dev[:, :L]
        out = torch.full((n, n + 3), 5.0, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st, mx = noalloc(dev, typ, model, RNJ_FASTDIST, out, stream)
        stream.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert st == 0
        if k == 1:  # the first call's set-up loaded every kernel: no device memory taken
            assert free_after >= free_before
        ref, rmx = existing(dev, typ, model, RNJ_FASTDIST)
        got = out[:, :n].cpu().numpy()
        d = ulp_diff(got, ref)
        assert d.max() <= 1 and (d == 1).sum() <= 2
        assert mx == rmx
        assert (out[:, n:] == 5.0).all()  # nothing written past the row
    # protein through the same array, twice in a row
    for seed in (3, 4):
        p = synth.tree_protein(257, 1500, seed=seed)
        dev = torch.from_numpy(p).cuda()
        out = torch.empty((257, 257), dtype=torch.float32, device="cuda")
        st, mx = noalloc(dev, RNJ_PROTEIN, RNJ_KIMURA, RNJ_FASTDIST, out)
        torch.cuda.synchronize()
        assert st == 0
        ref, rmx = existing(dev, RNJ_PROTEIN, RNJ_KIMURA, RNJ_FASTDIST)
        assert ulp_diff(out.cpu().numpy(), ref).max() <= 1 and mx == rmx


def test_noalloc_rejects_sizes_beyond_its_array():
    from rapidnj_b200 import _native
    from rapidnj_b200._native import RNJ_DNA, RNJ_FASTDIST, RNJ_KIMURA
    n, L = 6000, 10000  # 6000 x 10000 DNA needs ~23 MB of planes > 16 MiB
    dev = torch.zeros((n, 1), dtype=torch.uint8, device="cuda")
    out = torch.zeros((1, 1), dtype=torch.float32, device="cuda")
    st = _native.lib().rnj_distance_noalloc(ctypes.c_void_p(dev.data_ptr()), n, L, L, RNJ_DNA,
                                            RNJ_KIMURA, RNJ_FASTDIST, ctypes.c_void_p(out.data_ptr()),
                                            n, None, None)
    assert st == _native.RNJ_OK + 1  # RNJ_ERR_INVALID, before any kernel runs
    msg = _native.lib().rnj_last_error().decode()
    assert "16 MiB" in msg and "needs" in msg
