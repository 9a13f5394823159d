"""The served form: requests submitted concurrently, admitted by device memory,
batched while others run, give exactly the matrix each gives alone."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def request_mix(seed=0, count=24):
    from rapidnj_b200 import synth
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(16), np.log(700))))
        L = int(np.exp(rng.uniform(np.log(200), np.log(3000))))
        if k % 3 == 0:
            out.append((synth.iid_dna(n, L, seed=k), 0, "jc"))
        elif k % 3 == 1:
            out.append((synth.tree_protein(n, L, seed=k), 1, "kim"))
        else:
            out.append((synth.tree_dna(n, L, seed=k, mean_branch=0.1), 0, "kim"))
    return out


def test_served_results_equal_alone(ctx):
    from rapidnj_b200 import api
    reqs = request_mix(0)
    server = api.Server(0, max_batch=8)
    ids = [None] * len(reqs)

    def submit(part):
        for k in part:
            seqs, typ, model = reqs[k]
            ids[k] = server.submit(seqs, model, typ)

    threads = [threading.Thread(target=submit, args=(range(p, len(reqs), 2),)) for p in (0, 1)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for k, (seqs, typ, model) in enumerate(reqs):
        server.wait(ids[k])
        mat, lat = server.result(ctx, ids[k])
        alone = ctx.distance(ctx.alignment(seqs, typ), model)
        assert np.array_equal(mat.to_numpy(), alone.to_numpy())
        assert mat.max == alone.max
        assert lat > 0
        mat.close()
    st = server.stats()
    assert st["completed"] == len(reqs)
    assert st["bytes_in_use"] == 0
    server.close()


def test_served_admission_by_memory(ctx):
    """A budget that holds about two requests at a time still serves all, in order."""
    from rapidnj_b200 import api, synth
    seqs = [synth.tree_dna(256, 1000, seed=s) for s in range(6)]
    budget = 2 * (256 * 1000 + 256 * 4 * 1024 + 256 * 256 * 4 + 4096) + 1000
    server = api.Server(0, memory_budget=budget, max_batch=4)
    ids = [server.submit(s, "kim", 0) for s in seqs]
    for rid, s in zip(ids, seqs):
        server.wait(rid)
        m, _ = server.result(ctx, rid)
        ref = ctx.distance(ctx.alignment(s, 0), "kim").to_numpy()
        assert np.array_equal(m.to_numpy(), ref)
        m.close()
    server.close()


def test_served_rejects_requests_beyond_budget():
    from rapidnj_b200 import api, synth, RnjError
    server = api.Server(0, memory_budget=1 << 20)
    with pytest.raises(RnjError, match="budget"):
        server.submit(synth.tree_dna(512, 4000, seed=1), "kim", 0)
    server.close()


def test_served_beyond_the_staging_area(ctx, monkeypatch):
    # 36 requests of 9 MB each (324 MB) submitted at once: more than a 256 MiB
    # page-locked staging area (RNJ_SERVER_STAGING_MB; 1 GiB by default), so the
    # later ones are staged in pageable memory until extents are freed.  Every
    # result equals the plain call.
    from rapidnj_b200 import api, synth
    reqs = [(synth.tree_dna(1500, 6000, seed=100 + k, mean_branch=0.05), 0, "kim")
            if k % 2 == 0 else (synth.tree_protein(1500, 6000, seed=100 + k), 1, "kim")
            for k in range(36)]
    monkeypatch.setenv("RNJ_SERVER_STAGING_MB", "256")
    server = api.Server(0, max_batch=6)
    ids = [server.submit(s, m, t) for s, t, m in reqs]
    for k, (seqs, typ, model) in enumerate(reqs):
        server.wait(ids[k])
        m, _ = server.result(ctx, ids[k])
        got = m.to_numpy()
        m.close()
        aln = ctx.alignment(seqs, typ)
        ref = ctx.distance(aln, model)
        want = ref.to_numpy()
        ref.close()
        aln.close()
        assert np.array_equal(got.view(np.int32), want.view(np.int32))
    server.close()


def test_live_list_mixed_edges_and_generations(ctx):
    # Requests that join a running live kernel: tiny ones (n = 1, 2, L = 1),
    # saturated i.i.d. DNA under JC (the last tile's CTA applies the fix-up),
    # tree DNA and protein under Kimura, an 80-residue alphabet and -f DNA
    # (plain calls on the server's stream), in two waves so that the work
    # list starts a new generation of slots and items in between.  Each
    # result equals the plain call bit for bit, with the same maximum.
    from rapidnj_b200 import api, synth
    rng = np.random.default_rng(3)
    big = np.frombuffer(bytes(range(40, 120)), np.uint8)
    wave = []
    for k in range(40):
        kind = k % 8
        n = int(rng.integers(2, 900)) if kind else int(rng.integers(1, 4))
        L = int(rng.integers(1, 2500)) if kind != 1 else 1
        if kind in (0, 1, 2):
            wave.append((synth.iid_dna(max(n, 1), max(L, 1), seed=k), 0, "jc", True))
        elif kind == 3:
            wave.append((synth.tree_protein(n, L, seed=k), 1, "kim", True))
        elif kind == 4:
            s = big[rng.integers(0, big.size, (max(n, 2), 300))]
            wave.append((s, 1, "kim", True))
        elif kind == 5:
            wave.append((synth.tree_dna(n, L, seed=k, mean_branch=0.1), 0, "kim", False))
        else:
            wave.append((synth.tree_dna(n, L, seed=k, mean_branch=0.1), 0, "kim", True))
    server = api.Server(0, max_batch=16)
    for rnd in range(2):
        ids = [server.submit(s, m, t, fastdist=f) for s, t, m, f in wave]
        for rid, (seqs, typ, model, fast) in zip(ids, wave):
            server.wait(rid)
            m, lat = server.result(ctx, rid)
            got, gmax = m.to_numpy(), m.max
            m.close()
            aln = ctx.alignment(seqs, typ, fastdist=fast)
            ref = ctx.distance(aln, model)
            want, wmax = ref.to_numpy(), ref.max
            ref.close()
            aln.close()
            assert np.array_equal(got.view(np.int32), want.view(np.int32)) and gmax == wmax
            assert lat > 0
    st = server.stats()
    assert st["completed"] == 2 * len(wave) and st["bytes_in_use"] == 0
    server.close()
