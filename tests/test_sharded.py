"""The multi-GPU form's host logic, on the CPU: tile ranges and coordinates of the
shards (the C ABI's host arithmetic), and the two-step shard protocol with its one
MAX exchange run as two gloo ranks, each rank computing its tiles with the oracle.
The assembled matrix must equal the oracle's single-process matrix bit for bit."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

from conftest import ROOT

TILE = 128


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("full", [False, True])
def test_shard_ranges_cover_every_tile_once(full):
    from rapidnj_b200 import api
    for n in [1, 100, 128, 129, 1000, 10000, 50000]:
        nt = -(-n // TILE)
        total = nt * nt if full else nt * (nt + 1) // 2
        for ns in [1, 2, 3, 7, 8, 200]:
            prev, sizes = 0, []
            for s in range(ns):
                t0, t1, ntiles = api.shard_tiles(n, s, ns, full)
                assert ntiles == total and t0 == prev and t1 >= t0
                sizes.append(t1 - t0)
                prev = t1
            assert prev == total and max(sizes) - min(sizes) <= 1


def test_shard_rejects_bad_arguments():
    from rapidnj_b200 import api, RnjError
    for args in [(10, 2, 2), (10, -1, 2), (10, 0, 0), (-1, 0, 1)]:
        with pytest.raises(RnjError):
            api.shard_tiles(*args)
    with pytest.raises(RnjError):
        api.tile_coords(300, 6)  # 3 x 3 tiles: 6 triangle tiles, 0..5


@pytest.mark.parametrize("n", [1, 129, 1000, 5000])
def test_tile_coords_row_major_upper_triangle(n):
    from rapidnj_b200 import api
    nt = -(-n // TILE)
    tri = [(i, j) for i in range(nt) for j in range(i, nt)]
    for t, ij in enumerate(tri):
        assert api.tile_coords(n, t) == ij
    for t in range(nt * nt):
        assert api.tile_coords(n, t, full_rows=True) == divmod(t, nt)


def test_tile_coords_large_alignment():
    from rapidnj_b200 import api
    n = 200000
    nt = -(-n // TILE)
    start = lambda r: r * nt - r * (r - 1) // 2  # noqa: E731
    rng = np.random.default_rng(3)
    for r in list(rng.integers(0, nt, 200)) + [0, nt - 1]:
        r = int(r)
        for c in {r, nt - 1, r + (nt - r) // 2}:
            assert api.tile_coords(n, start(r) + c - r) == (r, c)


# ----------------------------------------------------------- two gloo ranks

class OracleShard:
    """A shard whose tiles come from the oracle: run() -> local max over its own
    pairs, finish(g) -> its pairs with saturated entries set to 2 * g, mirrored."""

    def __init__(self, raw, n, rank, world, full):
        from rapidnj_b200 import api
        self.raw, self.full = raw, full
        t0, t1, _ = api.shard_tiles(n, rank, world, full)
        own = np.zeros((n, n), bool)
        for t in range(t0, t1):
            ti, tj = api.tile_coords(n, t, full)
            own[ti * TILE:(ti + 1) * TILE, tj * TILE:(tj + 1) * TILE] = True
        i, j = np.indices((n, n))
        self.own = own & ((i != j) if full else (j > i))

    def run(self) -> float:
        v = self.raw[self.own]
        return float(max(0.0, v.max())) if v.size else 0.0

    def finish(self, g: float) -> None:
        out = np.where(self.own, self.raw, np.float32(0))
        out[self.own & (out == -1)] = np.float32(g) * np.float32(2)
        self.out = out if self.full else out + out.T


def _worker(rank, world, port, cases, q):
    import torch
    import torch.distributed as dist
    from rapidnj_b200 import sharded
    import oracle.oracle as O
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                                world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=60))
        for seqs, type_, model, naive, full in cases:
            n, L = seqs.shape
            cnt = O.counts(seqs, type_, naive, full)
            raw = O.raw_distances(cnt, L, type_, model, naive, False, full)
            sh = OracleShard(raw, n, rank, world, full)
            g = sharded.run_sharded(sh, None)
            total = torch.from_numpy(sh.out.copy())
            owners = torch.from_numpy((sh.own | (sh.own.T if not full else False)).astype(np.int32))
            dist.all_reduce(total, op=dist.ReduceOp.SUM)
            dist.all_reduce(owners, op=dist.ReduceOp.SUM)
            want, mx = O.matrix(cnt, L, type_, model, naive, False, full)
            off = ~np.eye(n, dtype=bool)
            assert (owners.numpy()[off] == 1).all(), "a pair owned by zero or two shards"
            assert g == mx, (g, mx)
            assert np.array_equal(total.numpy(), want)
        dist.barrier()
        dist.destroy_process_group()
        q.put((rank, "ok"))
    except BaseException as e:  # reported to the parent
        q.put((rank, repr(e)))


def test_two_ranks_assemble_the_single_process_matrix():
    import oracle.oracle as O
    from rapidnj_b200 import synth
    rng = np.random.default_rng(5)
    dna_short = rng.choice(np.frombuffer(b"ACGT-", np.uint8), size=(300, 24),
                           p=[0.24, 0.24, 0.24, 0.24, 0.04])
    dna_short[7, :] = ord("-")  # a sequence with no valid site: saturated against all
    prot = synth.iid_protein(260, 40, seed=2)
    cases = [
        (dna_short, O.DNA, O.KIMURA, False, False),   # many saturated pairs
        (dna_short, O.DNA, O.JC, False, False),
        (synth.tree_dna(290, 300, seed=4), O.DNA, O.KIMURA, False, False),
        (prot, O.PROTEIN, O.KIMURA, False, False),
        (dna_short[:200], O.DNA, O.KIMURA, True, True),  # -f full rows
        (dna_short[:100], O.DNA, O.KIMURA, False, False),  # one tile: rank 0 has none
    ]
    port = free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, cases, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert res == {0: "ok", 1: "ok"}, res
