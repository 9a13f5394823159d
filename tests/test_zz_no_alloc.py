"""rnj_distance_noalloc: distances for callers that cannot allocate device memory.

Who needs it: a process that owns the GPU through its own fixed memory pool (a
server that reserves device memory up front and forbids outside allocations),
or code that must not call cudaMalloc because it synchronises the device.  The
entry point takes the caller's device input, output and stream, and keeps its
intermediate buffers in one 16 MiB array built into the library.

The tests call it through the C ABI and compare each result with
rnj_distance_into, the entry point that allocates (and once with the oracle),
on calls made one after another, so that state left in the shared array by one
call (the running maximum, the saturation flags) would show in the next.  They
also check that the free device memory does not drop across a call, that sizes
beyond the array are refused, that a stream under capture is refused, and that
a bounded device wait that runs out is reported even without max_out.  The file
is collected last.
"""
import ctypes

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


def noalloc(seqs_dev, typ, model, flags, out, stream=None, want_max=True):
    from rapidnj_b200 import _native
    n, L = seqs_dev.shape
    m = ctypes.c_float()
    st = _native.lib().rnj_distance_noalloc(
        ctypes.c_void_p(seqs_dev.data_ptr()), n, L, seqs_dev.stride(0), typ, model, flags,
        ctypes.c_void_p(out.data_ptr()), out.stride(0),
        ctypes.c_void_p(stream.cuda_stream if stream is not None else 0),
        ctypes.byref(m) if want_max else None)
    return st, m.value


def existing(seqs_dev, typ, model, flags):
    from rapidnj_b200 import api
    ctx = api.Context(0)
    try:
        aln = ctx.alignment(seqs_dev, typ, fastdist=bool(flags & 1),
                            full_rows=bool(flags & api.RNJ_FULL_ROWS))
        n = seqs_dev.shape[0]
        out = torch.empty((n, n), dtype=torch.float32, device="cuda")
        mx = ctx.distance_into(aln, model, out, want_max=True)
        aln.close()
        return out.cpu().numpy(), mx
    finally:
        ctx.close()


def strided(seqs, pad=5):
    """The alignment on the device with a row stride wider than its rows."""
    n, L = seqs.shape
    dev = torch.zeros((n, L + pad), dtype=torch.uint8, device="cuda")
    dev[:, :L] = torch.from_numpy(seqs).cuda()
    return dev[:, :L]


def check_call(seqs, typ, model, flags, stream=None, want_max=True, memory_flat=True):
    """One no-allocation call: result equal to rnj_distance_into's, nothing written
    past the rows, no device memory taken."""
    n = seqs.shape[0]
    dev = strided(seqs)
    out = torch.full((n, n + 3), 5.0, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    st, mx = noalloc(dev, typ, model, flags, out, stream, want_max)
    free_after = torch.cuda.mem_get_info()[0]
    assert st == 0
    if memory_flat:
        assert free_after >= free_before
    ref, rmx = existing(dev, typ, model, flags)
    got = out[:, :n].cpu().numpy()
    d = ulp_diff(got, ref)
    assert d.max() <= 1 and (d == 1).sum() <= 2
    if want_max:
        assert mx == rmx
    assert (out[:, n:] == 5.0).all()  # nothing written past the row
    return got


def test_noalloc_matches_allocating_entry_on_calls_in_a_row():
    from rapidnj_b200 import synth
    from rapidnj_b200._native import (RNJ_DNA, RNJ_FASTDIST, RNJ_FULL_ROWS, RNJ_JC, RNJ_KIMURA,
                                      RNJ_PROTEIN)
    rng = np.random.default_rng(0)
    stream = torch.cuda.Stream()
    # call 1: many saturated pairs (unrelated short sequences), JC.  The first
    # call of the process on this device does the set-up (array address, kernel
    # loading), so its memory is not compared.
    a = np.frombuffer(b"ACGT", np.uint8)[rng.integers(0, 4, (300, 48))]
    check_call(a, RNJ_DNA, RNJ_JC, RNJ_FASTDIST, stream, memory_flat=False)
    # call 2: tree-evolved, no saturation, Kimura-2P, against the oracle too
    b = synth.tree_dna(700, 3000, seed=2, mean_branch=0.05)
    got = check_call(b, RNJ_DNA, RNJ_KIMURA, RNJ_FASTDIST, stream)
    ref, _ = oracle.distance_matrix(b, oracle.KIMURA, oracle.DNA)
    assert ulp_diff(got, ref).max() <= 1
    # calls 3, 4: the -f rules (naive counts), upper triangle and full rows;
    # lower-case and U sites make the naive counts asymmetric
    c = synth.tree_dna(260, 1000, seed=5, mean_branch=0.1)
    c[rng.random(c.shape) < 0.1] = ord("a")
    c[rng.random(c.shape) < 0.02] = ord("U")
    check_call(c, RNJ_DNA, RNJ_KIMURA, 0, stream)
    check_call(c, RNJ_DNA, RNJ_KIMURA, RNJ_FULL_ROWS, stream)
    # call 5: no max_out
    check_call(b, RNJ_DNA, RNJ_JC, RNJ_FASTDIST, stream, want_max=False)
    # calls 6, 7: protein after the DNA calls, twice in a row (20 residues)
    for seed in (3, 4):
        p = synth.tree_protein(257, 1500, seed=seed)
        check_call(p, RNJ_PROTEIN, RNJ_KIMURA, RNJ_FASTDIST)
    # call 8: an alphabet of more than 32 residue ranks (the widest plane layout)
    alpha = np.frombuffer(bytes(range(40, 120)), np.uint8)
    q = alpha[rng.integers(0, alpha.size, (150, 700))]
    q[rng.random(q.shape) < 0.05] = ord("-")
    got = check_call(q, RNJ_PROTEIN, RNJ_KIMURA, RNJ_FASTDIST)
    ref, _ = oracle.distance_matrix(q, oracle.KIMURA, oracle.PROTEIN)
    assert ulp_diff(got, ref).max() <= 1


def test_noalloc_rejects_sizes_beyond_its_array():
    from rapidnj_b200 import _native
    from rapidnj_b200._native import RNJ_DNA, RNJ_FASTDIST, RNJ_KIMURA
    dev = torch.zeros((1, 1), dtype=torch.uint8, device="cuda")
    out = torch.zeros((1, 1), dtype=torch.float32, device="cuda")
    # 6000 x 10000 DNA needs ~23 MB of planes > 16 MiB; 10 x 65281 columns is
    # beyond one counting pass.  Both are refused before any kernel runs (the
    # pointers are never read).
    for n, L, words in ((6000, 10000, ("16 MiB", "needs")), (10, 65281, ("65280",))):
        st = _native.lib().rnj_distance_noalloc(ctypes.c_void_p(dev.data_ptr()), n, L, L, RNJ_DNA,
                                                RNJ_KIMURA, RNJ_FASTDIST,
                                                ctypes.c_void_p(out.data_ptr()), n, None, None)
        assert st == _native.RNJ_ERR_INVALID
        msg = _native.lib().rnj_last_error().decode()
        assert all(w in msg for w in words), msg


def test_noalloc_refuses_a_capturing_stream():
    from rapidnj_b200 import _native, synth
    from rapidnj_b200._native import RNJ_DNA, RNJ_FASTDIST, RNJ_KIMURA
    seqs = torch.from_numpy(synth.tree_dna(64, 300, seed=1)).cuda()
    out = torch.zeros((64, 64), dtype=torch.float32, device="cuda")
    stream = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=stream):
        st, _ = noalloc(seqs, RNJ_DNA, RNJ_KIMURA, RNJ_FASTDIST, out, stream, want_max=False)
        out.add_(1.0)  # the capture itself stays valid
    assert st == _native.RNJ_ERR_UNSUPPORTED
    g.replay()
    torch.cuda.synchronize()
    assert (out == 1.0).all()


def test_noalloc_reports_a_timeout_without_max_out():
    """A bounded wait that runs out (the test switch makes the counting kernel
    wait on a barrier that nothing completes, for at most 1 ms) is returned as
    RNJ_ERR_TIMEOUT even when the caller asks for no maximum; the next call is
    correct again."""
    from rapidnj_b200 import _native, synth
    from rapidnj_b200._native import RNJ_DNA, RNJ_FASTDIST, RNJ_KIMURA
    lib = _native.lib()
    seqs = synth.tree_dna(200, 900, seed=9)
    dev = torch.from_numpy(seqs).cuda()
    out = torch.zeros((200, 200), dtype=torch.float32, device="cuda")
    lib.rnj_set_wait_limit(1000)
    lib.rnj_test_wait_on_unset_flag(1)
    try:
        st, _ = noalloc(dev, RNJ_DNA, RNJ_KIMURA, RNJ_FASTDIST, out, want_max=False)
    finally:
        lib.rnj_test_wait_on_unset_flag(0)
        lib.rnj_set_wait_limit(0)
    assert st == _native.RNJ_ERR_TIMEOUT
    check_call(seqs, RNJ_DNA, RNJ_KIMURA, RNJ_FASTDIST, want_max=False)
