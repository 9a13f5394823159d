"""The failure path of the counting kernels' bounded waits (rnj_set_wait_limit,
rnj_test_wait_on_unset_flag).

Every pipeline wait in the counting kernels is bounded.  When one runs out the
CTA stops, lets its own copies into shared memory land, frees its tensor memory
and sets the context's error word; the next call that waits for the GPU returns
RNJ_ERR_TIMEOUT.  The reference has no counterpart: its CPU code calls exit(1)
on errors (KimuraDistance.cpp:78-79).

The test switch makes the consumer warps wait first on a barrier that nothing
completes, under a 1 ms limit: the wait runs out, nothing faults or hangs.  The
same context must then compute the oracle's matrix again (tensor memory freed,
error word cleared).
"""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def ulp_max(a, b):
    a = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    a = np.where(a < 0, -(a & 0x7FFFFFFF), a)
    b = np.where(b < 0, -(b & 0x7FFFFFFF), b)
    return int(np.abs(a - b).max(initial=0))


@pytest.mark.parametrize("popcount", [False, True], ids=["tensor-cores", "bit-planes"])
def test_bounded_wait_runs_out_and_context_recovers(ctx, popcount):
    from rapidnj_b200 import _native, synth
    seqs = synth.tree_dna(300, 2000, seed=12, mean_branch=0.05)
    n = seqs.shape[0]
    out = torch.empty((n, n), dtype=torch.float32, device="cuda")
    lib = _native.lib()
    lib.rnj_set_wait_limit(1000)
    lib.rnj_test_wait_on_unset_flag(1)
    try:
        aln = ctx.alignment(seqs, oracle.DNA, popcount=popcount)
        with pytest.raises(_native.RnjError) as e:
            ctx.distance_into(aln, "kim", out, want_max=True)
        assert e.value.status == _native.RNJ_ERR_TIMEOUT
        # without a maximum the call does not wait: the sticky error word is
        # reported by the next synchronisation
        ctx.distance_into(aln, "kim", out)
        with pytest.raises(_native.RnjError) as e:
            ctx.synchronize()
        assert e.value.status == _native.RNJ_ERR_TIMEOUT
        aln.close()
    finally:
        lib.rnj_test_wait_on_unset_flag(0)
        lib.rnj_set_wait_limit(0)
    # the same context afterwards: correct distances, no stale error
    ctx.synchronize()
    aln = ctx.alignment(seqs, oracle.DNA, popcount=popcount)
    mx = ctx.distance_into(aln, "kim", out, want_max=True)
    aln.close()
    ref, rmx = oracle.distance_matrix(seqs, oracle.KIMURA, oracle.DNA)
    assert ulp_max(out.cpu().numpy(), ref) <= 1 and mx == rmx
