#!/usr/bin/env python
"""Benchmark: pair-column comparisons per second of the all-pairs distance path.

One unit = one (i < j, column) comparison; an alignment of n sequences and L
columns is n (n - 1) / 2 * L units.  A step is one pass of the path over one
alignment: pack the resident bytes (FP4 features for the tensor cores, or bit
planes), count every pair, apply the transform, post-process (mirror, diagonal,
saturation fix-up).

Default workload (one B200): DNA Kimura-2P, 10,000 x 10,000, tree-evolved
synthetic alignment.  Output: one JSON line on rank 0.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...   (the reference's threaded CPU path)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (generator, n, L, type, model)
    "dna-k2p-10000x10000": ("tree_dna", 10000, 10000, "dna", "kim"),
    "dna-jc-512x2000": ("iid_dna", 512, 2000, "dna", "jc"),
    "dna-k2p-50000x1000": ("tree_dna", 50000, 1000, "dna", "kim"),
    "protein-kimura-5000x1500": ("tree_protein", 5000, 1500, "protein", "kim"),
    # the same kernel as the default workload at a size an ncu --set full capture
    # finishes quickly (inputs + planes + output ~ 0.2 GB, larger than L2)
    "dna-k2p-4096x10000": ("tree_dna", 4096, 10000, "dna", "kim"),
}
DEFAULT = "dna-k2p-10000x10000"
# The other single-GPU configurations, measured in the default run beside it.
OTHER_CONFIGS = ("dna-jc-512x2000", "dna-k2p-50000x1000", "protein-kimura-5000x1500")
# Algorithmic integer operations per pair per 32-column word of the bit-plane
# counting kernel, (POPC, LOP3) for each (type, model): its roofline when the
# bit planes are used (--popcount, or protein alphabets of more than 31 residues).
OPS_PER_WORD = {("dna", "kim"): (3, 4), ("dna", "jc"): (2, 4), ("protein", "kim"): (2, 7),
                ("protein", "jc"): (2, 7)}


def make_alignment(name: str, seed: int = 0) -> np.ndarray:
    from rapidnj_b200 import synth
    gen, n, L, _, _ = WORKLOADS[name]
    return getattr(synth, gen)(n, L, seed=seed)


def residue_ranks(seqs: np.ndarray) -> int:
    """Distinct residue bytes of a protein alignment (gap bytes of the reference
    loader's resolveChar excluded): the one-hot feature blocks it takes."""
    gaps = set(b"-.XxzZbBJj?")
    return sum(1 for c in np.unique(seqs) if int(c) not in gaps)


def units(n: int, L: int) -> float:
    return n * (n - 1) / 2.0 * L


# ------------------------------------------------------------------ clocks

class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            # nvidia-smi needs a moment to start: begin timing once it samples.
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.lines.clear()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- CPU baseline

def cpu_reference(seqs: np.ndarray, model: str, type_: str, warmup: int, steps: int,
                  budget_s: float = 12.0):
    """The reference's threaded SSE path (oracle/_ref/ref_harness, built from the
    reference sources) on all host cores, on a bounded sample of the workload:
    the first n' sequences, n' chosen so one call takes about budget_s."""
    from oracle import oracle
    from rapidnj_b200 import synth
    if not oracle.ref_available():
        return None
    cores = os.cpu_count() or 1
    n, L = seqs.shape
    t = "d" if type_ == "dna" else "p"

    def run(rows: int, w: int, s: int):
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "sample.fa")
            synth.write_fasta(path, seqs[:rows])
            p = subprocess.run([oracle.REF_HARNESS, "bench", path, "fa", t, "1", model, str(cores),
                                str(w), str(s)], check=True, capture_output=True, text=True)
            return json.loads(p.stdout.strip().splitlines()[-1])["step_s"]

    probe_rows = min(n, 1024)
    probe = run(probe_rows, 0, 1)[0]
    rate = units(probe_rows, L) / max(probe, 1e-6)
    rows = n
    if units(n, L) / rate > budget_s:
        rows = int((2.0 * budget_s * rate / L) ** 0.5)
        rows = max(probe_rows, min(n, rows))
    times = run(rows, warmup, steps)
    mean = sum(times) / len(times)
    return {"value": units(rows, L) / mean, "unit": "pair-columns/s", "cores": cores,
            "kind": "reference",
            "sample": f"first {rows} of {n} sequences x {L} columns, {len(times)} timed call(s) "
                      f"of the reference driver (oracle/_ref/ref_harness, g++ -O3 -msse2, "
                      f"{cores} threads)",
            "step_s": times}


# ------------------------------------------------------------------ GPU arm

def measure_workload(name: str, steps: int, warmup: int, rank: int = 0, world: int = 1,
                     local_rank: int = 0, popcount: bool = False, with_e2e: bool = True,
                     clocks: bool = True, roofline: bool = True):
    """One workload through the library: W warm-up steps, then K timed steps
    (CUDA events on the library's stream, a 256 MiB buffer written between
    steps so that L2 starts cold).  Returns the figures of the JSON line."""
    import torch
    import torch.distributed as dist
    from rapidnj_b200 import api, sharded

    gen, n, L, type_, model = WORKLOADS[name]
    seqs = make_alignment(name, seed=0)
    typ = 0 if type_ == "dna" else 1
    ctx = api.Context(local_rank)
    ctx.set_profiling(True)
    stream = torch.cuda.ExternalStream(ctx.stream)
    d_chars = torch.from_numpy(seqs).cuda(local_rank)
    out = torch.empty((n, n), dtype=torch.float32, device=f"cuda:{local_rank}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")  # > 126 MB L2
    torch.cuda.synchronize()

    def step():
        aln = ctx.alignment(d_chars, typ, popcount=popcount)
        if world > 1:
            # this rank's contiguous range of tiles; one float MAX all-reduce
            sh = api.Shard(ctx, aln, model, rank, world, out)
            sharded.run_sharded(sh, None, local_rank)
            sh.close()
        else:
            ctx.distance_into(aln, model, out)
        aln.close()

    # The clock record covers the warm-up and the timed steps (the timed region
    # alone can be shorter than one nvidia-smi sample).
    sampler = ClockSampler(local_rank).start() if clocks else None
    for _ in range(warmup):
        step()
    ctx.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    total_ms, count_ms, post_ms, pack_ms = 0.0, [], [], []
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()  # L2 flush between timed steps (outside the events)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        b.synchronize()
        total_ms += a.elapsed_time(b)
        st = ctx.stage_times()
        count_ms.append(st[1])
        post_ms.append(st[2])
        pack_ms.append(st[0])
    torch.cuda.synchronize()
    clk = sampler.stop() if sampler else None
    if world > 1:
        t = torch.tensor([total_ms], device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    ms_per_step = total_ms / steps
    W = units(n, L)  # the whole matrix, whatever the number of ranks
    # this rank's share of the tiles (all of them on one GPU)
    t0, t1, ntiles = api.shard_tiles(n, rank, world)
    share = (t1 - t0) / ntiles
    mean = lambda x: sum(x) / len(x)  # noqa: E731
    tc = not popcount and (type_ == "dna" or residue_ranks(seqs) <= 31)
    # the fused kernel unless the tuner's entry for this bucket chose the
    # two-kernel form
    entry = api.tune_get(n, L, type_)
    fused = tc and L <= 65535 and (entry is None or entry.tc_epilogue == 0)
    result = {"ms_per_step": ms_per_step, "value": W / (ms_per_step * 1e-3), "clocks": clk,
              "stages_ms": {"pack": mean(pack_ms),
                            "count_and_transform" if fused else "count": mean(count_ms),
                            "fixup" if fused else "transform_and_fixup": mean(post_ms)},
              "kernel": "tcgen05" if tc else "popcount",
              # per step: (protein: presence scan) + pack + counting kernel(s) + fix-up
              "gpu_launches_per_step": (1 if type_ == "protein" else 0) + 3 +
                                       (0 if (fused or not tc) else 1)}

    if rank == 0 and roofline:
        cnt = mean(count_ms)
        if tc:
            # tcgen05 kernel, against the FP4 tensor pipe measured live on this
            # device (back-to-back kind::mxf4 MMAs, rnj_probe_tc_peak): DNA 4 FP4
            # MACs (8 flops) per pair-column; protein 1 + R MACs (valid + one-hot
            # of R residue ranks).
            fpc = 8 if type_ == "dna" else 2 * (1 + residue_ranks(seqs))
            pipe = ctx.probe_tc_peak()
            bf16x4, bf16_src = fp4_from_bf16()
            achieved = fpc * units(n, L) * share / (cnt * 1e-3)
            kname = "tc_fused_kernel" if fused else "tc_batch_kernel"
            result["roofline"] = {
                "bound": "tensor", "achieved": achieved / 1e12, "peak": pipe / 1e12,
                "unit": "TFLOP/s", "frac": achieved / pipe,
                "format": "fp4 e2m1 operands (tcgen05 kind::mxf4), f32 sums",
                "peak_source": "FP4 tensor pipe measured on this device in this run "
                               "(rnj_probe_tc_peak: back-to-back 128x128x64 kind::mxf4 MMAs "
                               "on every SM); 4 x measured dense bf16 beside it",
                "peak_4x_bf16": bf16x4 / 1e12, "frac_of_4x_bf16": achieved / bf16x4,
                "peak_4x_bf16_source": bf16_src,
                "traffic": traffic_from_profiles(kname, name), "kernel": kname, "kernel_ms": cnt,
                "flops_per_pair_column": fpc,
                "kernel_includes": ("counts, exact transform and the matrix stores" if fused
                                    else "counts (the transform is a second kernel)"),
            }
        else:
            # Bit-plane popcount kernel: bound by the POPC pipe, against the
            # POPC peak measured on this device.
            popc_peak, lop3_peak = ctx.probe_int_peaks()
            popc_w, lop3_w = OPS_PER_WORD[(type_, model)]
            words = units(n, L) * share / 32.0
            achieved = popc_w * words / (cnt * 1e-3)
            result["roofline"] = {
                "bound": "int", "pipe": "POPC", "achieved": achieved / 1e12,
                "peak": popc_peak / 1e12, "unit": "Tops/s", "frac": achieved / popc_peak,
                "traffic": traffic_from_profiles(
                    "count_batch_kernel" if world > 1 else "count_tiles_kernel", name),
                "kernel": "count_batch_kernel" if world > 1 else "count_tiles_kernel",
                "kernel_ms": cnt,
                "lop3_frac": (lop3_w * words / (cnt * 1e-3)) / lop3_peak,
                "peak_source": "rnj_probe_int_peaks, measured on this device in this run",
                "ops_per_pair_word": {"popc": popc_w, "lop3": lop3_w},
            }
    if with_e2e:
        if world > 1:
            result["e2e"] = run_e2e_sharded(ctx, seqs, typ, model, steps, popcount, rank, world,
                                            local_rank)
        elif rank == 0:
            result["e2e"] = run_e2e(ctx, seqs, typ, model, steps, popcount)
    del out, flush, d_chars
    ctx.close()
    torch.cuda.empty_cache()
    return result


def run_e2e(ctx, seqs, typ, model, steps, popcount=False):
    """The same metric through the host-facing C ABI call (rnj_distance_matrix_host):
    page-locked host bytes in, the caller's page-locked host n x n float matrix
    out; upload, pack, distances and the device-to-host copy of the whole matrix
    inside the timed region."""
    import torch
    n, L = seqs.shape
    pinned = torch.from_numpy(seqs).pin_memory()
    host = pinned.numpy()
    # the caller's result matrix: page-locked host memory, allocated once
    out = torch.empty((n, n), dtype=torch.float32).pin_memory().numpy()
    steps = max(1, min(steps, 10))
    ctx.distance_matrix_host(host, model, typ, popcount=popcount, out=out)  # warm-up
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        ctx.distance_matrix_host(host, model, typ, popcount=popcount, out=out)
        times.append(time.perf_counter() - t0)
    # median step: the host side shares its cores with other jobs on the machine
    med = statistics.median(times)
    return {"value": units(n, L) / med, "unit": "pair-columns/s", "h2d_bytes_per_step": n * L,
            "d2h_bytes_per_step": n * n * 4, "ms_per_step": med * 1e3,
            "mean_ms": 1e3 * sum(times) / len(times), "steps": steps,
            "call": "rnj_distance_matrix_host"}


def run_e2e_sharded(ctx, seqs, typ, model, steps, popcount, rank, world, local_rank):
    """The multi-GPU end to end: every rank uploads the host alignment (pinned),
    packs it, computes its tiles, joins the one MAX all-reduce, applies the cap
    and copies its own tiles into pinned host memory.  Time = max over ranks."""
    import torch
    import torch.distributed as dist
    from rapidnj_b200 import api, sharded
    n, L = seqs.shape
    pinned = torch.from_numpy(seqs).pin_memory()
    host = torch.empty((n, n), dtype=torch.float32).pin_memory().numpy()
    stream = torch.cuda.ExternalStream(ctx.stream)
    steps = max(1, min(steps, 5))

    def once():
        with torch.cuda.stream(stream):
            d = pinned.to(f"cuda:{local_rank}", non_blocking=True)
        aln = ctx.alignment(d, typ, popcount=popcount)
        sh = api.Shard(ctx, aln, model, rank, world)
        sharded.run_sharded(sh, None, local_rank)
        nbytes = sh.copy_tiles(host)
        sh.close()
        aln.close()
        return nbytes

    once()  # warm-up
    dist.barrier()
    times, d2h = [], 0
    for _ in range(steps):
        t0 = time.perf_counter()
        d2h = once()
        times.append(time.perf_counter() - t0)
    t = torch.tensor([sum(times) / len(times), float(d2h)], dtype=torch.float64,
                     device=f"cuda:{local_rank}")
    tot = t.clone()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    mean = float(t[0].item())
    return {"value": units(n, L) / mean, "unit": "pair-columns/s",
            "h2d_bytes_per_step": n * L * world, "d2h_bytes_per_step": int(tot[1].item()),
            "ms_per_step": mean * 1e3, "steps": steps,
            "call": "rnj_aln_from_device + rnj_shard_run/finish + rnj_shard_copy_tiles per rank"}


def run_batched(args, local_rank: int = 0, count: int = 256):
    """The mixed workload (N ~ U[32, 2048], L ~ U[300, 5000], 70 % tree DNA
    Kimura-2P, 30 % tree protein Kimura): plain per-request calls (pack +
    rnj_distance_into per alignment) against one batched pass (pack each, one
    graph-captured persistent launch over all tiles).  Inputs resident; outputs
    preallocated; the matrices of both must be identical."""
    import torch
    from rapidnj_b200 import api, synth
    mix = synth.batch_mix(count, seed=0)
    ctx = api.Context(local_rank)
    dev = [torch.from_numpy(s).cuda(local_rank) for _, s in mix]
    typ = [0 if k == "dna" else 1 for k, _ in mix]
    outs_a = [torch.empty((s.shape[0], s.shape[0]), device=f"cuda:{local_rank}") for _, s in mix]
    outs_b = [torch.empty((s.shape[0], s.shape[0]), device=f"cuda:{local_rank}") for _, s in mix]
    W = sum(units(*s.shape) for _, s in mix)
    stream = torch.cuda.ExternalStream(ctx.stream)
    tiles = sum(((s.shape[0] + 127) // 128) * ((s.shape[0] + 127) // 128 + 1) // 2 for _, s in mix)
    batch = api.Batch(ctx, max_alignments=count, max_tiles=tiles + 16)

    def plain():
        for d, t, o in zip(dev, typ, outs_a):
            a = ctx.alignment(d, t)
            ctx.distance_into(a, "kim", o)
            a.close()

    def batched():
        batch.add_many(dev, typ, ["kim"] * count, outs=outs_b)
        batch.run()
        batch.clear()

    def timed(fn, steps):
        total = 0.0
        for _ in range(steps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            total += a.elapsed_time(b)
        return total / steps

    for _ in range(max(1, args.warmup)):
        plain()
        batched()
    ctx.synchronize()
    steps = max(1, min(args.steps, 5))
    t_plain = timed(plain, steps)

    def tuned_pass():
        batched()  # untimed: the first run after a switch
        return timed(batched, steps)

    def untuned_pass():
        batched()
        return timed(batched, steps), batch.tuning()

    # tuned and untuned passes alternate (three each), so that neither gains
    # from running later; the line's figure is the tuned mean
    t_tuned, t_untuned = [], []
    identical = True
    for _ in range(3):
        t_tuned.append(tuned_pass())
        # launch shape of the batched pass: each alignment's tile-order band
        # from its bucket's tuned entry, the ring depth from the bucket with
        # the most work
        depth, tuned = batch.tuning()
        identical = identical and all(torch.equal(x, y) for x, y in zip(outs_a, outs_b))
        t, (depth0, _) = without_tuning(untuned_pass)
        t_untuned.append(t)
        identical = identical and all(torch.equal(x, y) for x, y in zip(outs_a, outs_b))
    t_batch = sum(t_tuned) / len(t_tuned)
    t_untuned = sum(t_untuned) / len(t_untuned)
    t_tuned_mean = t_batch
    batch.close()
    ctx.close()
    return {"value": W / (t_batch * 1e-3), "unit": "pair-columns/s", "ms_per_step": t_batch,
            "plain_value": W / (t_plain * 1e-3), "plain_ms_per_step": t_plain,
            "speedup_vs_plain": t_plain / t_batch, "identical_to_plain": identical,
            "shapes": {"source": "autotuner table " + str(tune_table_source()),
                       "tuned_alignments": tuned, "ring_depth": depth,
                       "tile_shape": "128 x 128 pairs (the tcgen05 M and the shared tile order)",
                       "tuned_ms_per_step": t_tuned_mean, "untuned_ms_per_step": t_untuned,
                       "untuned_ring_depth": depth0,
                       "timing": "tuned and untuned passes alternated, three each, each "
                                 "after one untimed run"},
            "alignments": count, "tiles": tiles, "pair_columns": W,
            "workload": "256 alignments, N~U[32,2048], L~U[300,5000], 70% DNA K2P / 30% "
                        "protein Kimura, tree-evolved, seed 0"}


def run_served(args, local_rank: int = 0, rate: float = 1000.0, seconds: float = 3.0,
               pool_size: int = 64):
    """The served workload: requests with N log-uniform in [16, 4096] and L
    log-uniform in [200, 8000], 50/50 DNA Jukes-Cantor / protein Kimura
    (i.i.d. residues, 5 % gaps; a pool of seeded alignments submitted in turn).
    (1) Poisson arrivals at `rate` requests/s for `seconds`: p50/p99 latency from
    submit to the matrix complete on the device; (2) all requests at once:
    saturation throughput; (3) the same requests as plain per-request calls."""
    import threading
    import torch
    from rapidnj_b200 import api, synth
    sizes = synth.served_sizes(pool_size, seed=0)
    pool = []
    for k, (kind, n, L) in enumerate(sizes):
        if kind == "dna":
            pool.append((synth.iid_dna(n, L, seed=k), 0, "jc"))
        else:
            pool.append((synth.iid_protein(n, L, seed=k), 1, "kim"))
    ctx = api.Context(local_rank)
    server = api.Server(local_rank, max_batch=256)

    def drive(count, arrivals):
        ids, lat = [], []
        done = threading.Event()

        def collect():
            for k in range(count):
                while len(ids) <= k:
                    time.sleep(0.0001)
                server.wait(ids[k])
                m, ms = server.result(ctx, ids[k])
                lat.append(ms)
                m.close()
            done.set()

        th = threading.Thread(target=collect)
        th.start()
        t0 = time.perf_counter()
        for k in range(count):
            if arrivals is not None:
                delay = t0 + arrivals[k] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
            seqs, typ, model = pool[k % pool_size]
            ids.append(server.submit(seqs, model, typ))
        th.join()
        wall = time.perf_counter() - t0
        work = sum(units(*pool[k % pool_size][0].shape) for k in range(count))
        return lat, work, wall

    # warm-up
    drive(pool_size, None)
    # each request alone (submitted after the previous one completed): the
    # latency it has without other requests in the server
    alone = []
    for seqs, typ, model in pool:
        time.sleep(0.002)
        rid = server.submit(seqs, model, typ)
        server.wait(rid)
        m, ms = server.result(ctx, rid)
        m.close()
        alone.append(ms)
    rng = np.random.default_rng(1)
    count = int(rate * seconds)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=count))
    lat, work, wall = drive(count, arrivals)
    slowdown = np.array([lat[k] / alone[k % pool_size] for k in range(count)])
    sat_lat, sat_work, sat_wall = drive(4 * pool_size, None)
    # plain per-request calls on the same requests
    stream = torch.cuda.ExternalStream(ctx.stream)
    t0 = time.perf_counter()
    plain_work = 0.0
    for k in range(2 * pool_size):
        seqs, typ, model = pool[k % pool_size]
        a = ctx.alignment(seqs, typ)
        m = ctx.distance(a, model)
        a.close()
        m.close()
        plain_work += units(*seqs.shape)
    ctx.synchronize()
    plain_wall = time.perf_counter() - t0
    server.close()
    ctx.close()
    lat = np.array(lat)
    return {"rate_req_per_s": rate, "requests": count,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "p99_over_p50": float(np.percentile(lat, 99) / np.percentile(lat, 50)),
            "alone_p50_ms": float(np.percentile(alone, 50)),
            "alone_p99_ms": float(np.percentile(np.array(alone)[[k % pool_size
                                                                for k in range(count)]], 99)),
            "slowdown_p50": float(np.percentile(slowdown, 50)),
            "slowdown_p99": float(np.percentile(slowdown, 99)),
            "slowdown_note": "a request's latency in the mix / its latency submitted alone",
            "mean_ms": float(lat.mean()), "throughput": work / wall,
            "saturation_throughput": sat_work / sat_wall,
            "saturation_p50_ms": float(np.percentile(sat_lat, 50)),
            "plain_throughput": plain_work / plain_wall,
            "saturation_vs_plain": (sat_work / sat_wall) / (plain_work / plain_wall),
            "unit": "pair-columns/s",
            "workload": "N log-uniform [16,4096], L log-uniform [200,8000], 50/50 DNA JC / "
                        "protein Kimura, i.i.d. residues with 5% gaps, pool of 64 seeded "
                        "alignments, host input (H2D inside)"}


def run_bootstrap(args, local_rank: int = 0, n: int = 2000, L: int = 2000, R: int = 100):
    """Bootstrap replicates (rapidNJ -b): R replicates of a resident DNA K2P
    alignment (tree-evolved, n x L) with seeded random columns, by rnj_bootstrap
    (gather + batches) against one plain call per replicate on bytes gathered on
    the device; identical matrices required."""
    import torch
    from rapidnj_b200 import api, synth
    ctx = api.Context(local_rank)
    dev = f"cuda:{local_rank}"
    seqs = torch.from_numpy(synth.tree_dna(n, L, seed=3)).to(dev)
    cols = np.random.default_rng(0).integers(0, L, size=(R, L))
    cols_t = torch.from_numpy(cols).to(dev)
    outs_a = [torch.empty((n, n), device=dev) for _ in range(R)]
    outs_b = [torch.empty((n, n), device=dev) for _ in range(R)]

    def plain():
        for r in range(R):
            a = ctx.alignment(seqs[:, cols_t[r]].contiguous(), 0)
            ctx.distance_into(a, "kim", outs_a[r])
            a.close()
        ctx.synchronize()

    def boot():
        ctx.bootstrap(seqs, cols, 0, "kim", outs=outs_b)

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    for fn in (plain, boot):
        fn()
    tp = statistics.median(timed(plain) for _ in range(3))
    tb = statistics.median(timed(boot) for _ in range(3))
    W = R * units(n, L)
    identical = all(torch.equal(x, y) for x, y in zip(outs_a, outs_b))
    ctx.close()
    return {"value": W / tb, "unit": "pair-columns/s", "ms": 1e3 * tb,
            "plain_ms": 1e3 * tp, "speedup_vs_plain": tp / tb,
            "identical_to_plain": identical,
            "workload": f"{R} replicates of DNA K2P {n} x {L} (tree-evolved), seeded columns"}


def run_nj_init(args, local_rank: int = 0, n: int = 10000, L: int = 10000):
    """rapidNJ's NJ set-up (rapidNJ::initialize: separation sums, redundant rows,
    sorted rows) by rnj_nj_init over the device matrix of the DNA K2P n x L
    workload, against the reference's own initialize() (oracle/_ref/nj_harness,
    one host thread, as in the reference) on the same matrix when built."""
    import torch
    from rapidnj_b200 import api, synth
    ctx = api.Context(local_rank)
    dev = f"cuda:{local_rank}"
    seqs = synth.tree_dna(n, L, seed=0)
    aln = ctx.alignment(torch.from_numpy(seqs).to(dev), 0)
    m = torch.empty((n, n), dtype=torch.float32, device=dev)
    ctx.distance_into(aln, "kim", m)
    aln.close()
    ctx.synchronize()
    sorted_out = torch.empty((n, n - 1, 2), dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    ts = []
    for r in range(6):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = ctx.nj_init(m, sorted_out=sorted_out)
        t1 = time.perf_counter()
        if r >= 1:
            ts.append(t1 - t0)
    out = {"ms": 1e3 * statistics.median(ts), "n": n,
           "redundant_rows": int((res["index_to_id"] == -1).sum()),
           "sorted_entries": int(res["row_lengths"].sum()),
           "workload": f"rapidNJ initialize() over the DNA K2P {n} x {n} matrix of the {n} x {L} "
                       "tree-evolved alignment (device-resident), sorted rows kept on the device"}
    if not args.no_cpu_baseline:
        try:
            sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
            from oracle import oracle
            if os.path.exists(os.path.join(oracle.REF_DIR, "nj_harness")):
                _, info = oracle.ref_nj_init(m.cpu().numpy(), 0, reps=1, want=False)
                out["cpu_reference_ms"] = 1e3 * info["init_s"][0]
                out["cpu_reference"] = ("rapidNJ::initialize from the reference sources "
                                        "(oracle/_ref/nj_harness), 1 thread, same matrix")
                out["speedup_vs_cpu_reference"] = out["cpu_reference_ms"] / out["ms"]
        except Exception as e:  # the baseline is reported, never required
            out["cpu_reference_error"] = str(e)[:200]
    ctx.close()
    return out


def run_parse(args, local_rank: int = 0):
    """Reading the workload's alignment from a FASTA file (60 columns a line): the
    device reader (rnj_msa_read_device: page-locked threaded read, parse on the
    GPU) against the host reader (rnj_msa_read), both through the C ABI with the
    file in the page cache; and file -> distance matrix in page-locked host memory
    through the device reader (read, pack, distances, one download)."""
    import ctypes
    import torch
    from rapidnj_b200 import _native as N
    from rapidnj_b200 import api, synth
    _, n, L, type_, model = WORKLOADS[args.workload]
    seqs = make_alignment(args.workload)
    lib = N.lib()
    dev = f"cuda:{local_rank}"
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "aln.fa").encode()
        synth.write_fasta(path.decode(), seqs, width=60)
        size = os.path.getsize(path)
        ctx = api.Context(local_rank)

        def read(device: bool):
            h = ctypes.c_void_p()
            t0 = time.perf_counter()
            if device:
                N.check(lib.rnj_msa_read_device(ctx.handle, path, b"fa", ctypes.byref(h)))
            else:
                N.check(lib.rnj_msa_read(path, b"fa", ctypes.byref(h)))
            return h, time.perf_counter() - t0

        out_d = torch.empty((n, n), dtype=torch.float32, device=dev)
        out_h = torch.empty((n, n), dtype=torch.float32).pin_memory()

        def file_to_matrix():
            t0 = time.perf_counter()
            h, _ = read(True)
            p, ld = ctypes.c_void_p(), ctypes.c_size_t()
            N.check(lib.rnj_msa_device_chars(h, ctypes.byref(p), ctypes.byref(ld)))
            nn, LL, tt = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            N.check(lib.rnj_msa_info(h, ctypes.byref(nn), ctypes.byref(LL), ctypes.byref(tt)))
            a = ctypes.c_void_p()
            N.check(lib.rnj_aln_from_device(ctx.handle, p, nn.value, LL.value, ld.value, tt.value,
                                            N.RNJ_FASTDIST, ctypes.byref(a)))
            N.check(lib.rnj_distance_into(ctx.handle, a, api.MODELS[model],
                                          ctypes.c_void_p(out_d.data_ptr()), n, None))
            lib.rnj_aln_destroy(a)
            ctx.synchronize()
            out_h.copy_(out_d)
            torch.cuda.synchronize()
            lib.rnj_msa_destroy(h)
            return time.perf_counter() - t0

        for dv in (True, False):  # warm-up: page cache, page-locked buffer
            h, _ = read(dv)
            lib.rnj_msa_destroy(h)
        tdv, thv = [], []
        for _ in range(4):
            h, t = read(True)
            lib.rnj_msa_destroy(h)
            tdv.append(t)
            h, t = read(False)
            lib.rnj_msa_destroy(h)
            thv.append(t)
        file_to_matrix()
        tf = statistics.median(file_to_matrix() for _ in range(3))
        ctx.close()
    return {"file_mb": size / 1e6, "device_reader_ms": 1e3 * statistics.median(tdv),
            "host_reader_ms": 1e3 * statistics.median(thv),
            "speedup_vs_host_reader": statistics.median(thv) / statistics.median(tdv),
            "file_to_host_matrix_ms": 1e3 * tf,
            "workload": f"FASTA file of the {args.workload} alignment, 60 columns a line, "
                        "names s0.., file in the page cache"}


def run_text(args, local_rank: int = 0):
    """The "-o m" text of the workload's distance matrix (rapidNJ's
    printDistanceMatrix): rnj_write_matrix_text_device (formatted on the device)
    against rnj_write_matrix_text (host, all cores), files compared byte for byte."""
    import torch
    from rapidnj_b200 import api
    _, n, L, type_, model = WORKLOADS[args.workload]
    seqs = make_alignment(args.workload)
    dev = f"cuda:{local_rank}"
    ctx = api.Context(local_rank)
    aln = ctx.alignment(torch.from_numpy(np.ascontiguousarray(seqs)).to(dev), api.TYPES[type_])
    m = torch.empty((n, n), dtype=torch.float32, device=dev)
    ctx.distance_into(aln, model, m)
    aln.close()
    ctx.synchronize()
    names = [f"s{i}" for i in range(n)]
    with tempfile.TemporaryDirectory() as td:
        pd, ph = os.path.join(td, "d.txt"), os.path.join(td, "h.txt")
        api.write_matrix_text_device(ctx, pd, names, m)  # warm-up
        tdv = []
        for _ in range(3):
            t0 = time.perf_counter()
            api.write_matrix_text_device(ctx, pd, names, m)
            tdv.append(time.perf_counter() - t0)
        host = m.cpu().numpy()
        t0 = time.perf_counter()
        api.write_matrix_text(ph, names, host)
        th = time.perf_counter() - t0
        size = os.path.getsize(pd)
        with open(pd, "rb") as a, open(ph, "rb") as b:
            same = a.read() == b.read()
    ctx.close()
    return {"text_mb": size / 1e6, "device_writer_ms": 1e3 * statistics.median(tdv),
            "host_writer_ms": 1e3 * th, "speedup_vs_host_writer": th / statistics.median(tdv),
            "identical": same, "host_threads": os.cpu_count(),
            "workload": f"-o m text of the {args.workload} matrix into a file (page cache)"}


def tune_table_source():
    """The tuning table the library read at its first lookup (as it chooses:
    RNJ_TUNE_CACHE, else the table shipped beside librnjgpu.so unless
    RNJ_NO_TUNE_TABLE is set), relative to the repository when inside it."""
    p = os.environ.get("RNJ_TUNE_CACHE")
    if not p:
        off = os.environ.get("RNJ_NO_TUNE_TABLE", "")
        p = None if (off and off != "0") else os.path.join(ROOT, "rapidnj_b200", "tune_b200.txt")
    if not p or not os.path.exists(p):
        return None
    p = os.path.abspath(p)
    return os.path.relpath(p, ROOT) if p.startswith(ROOT + os.sep) else p


def without_tuning(fn):
    """fn() with the tuning table emptied (every bucket at the library's
    defaults), the table restored afterwards."""
    import tempfile
    from rapidnj_b200 import api
    fd, path = tempfile.mkstemp(suffix=".tune")
    os.close(fd)
    try:
        api.tune_save(path)
        api.tune_clear()
        return fn()
    finally:
        api.tune_load(path)
        os.unlink(path)


def tuning_report(name, steps, local_rank, popcount, tuned_ms):
    """The plain workload at the tuned choice of its bucket against the
    library's defaults (fewer steps, no roofline or end-to-end run)."""
    from rapidnj_b200 import api
    _, n, L, type_, _ = WORKLOADS[name]
    entry = api.tune_get(n, L, type_)
    rep = {"table": tune_table_source(), "entry": entry.as_dict() if entry else None,
           "tuned_ms_per_step": tuned_ms}
    if entry is None:
        rep["default_ms_per_step"] = tuned_ms
        return rep
    r = without_tuning(lambda: measure_workload(name, max(3, min(steps, 20)), 3,
                                                local_rank=local_rank, popcount=popcount,
                                                with_e2e=False, clocks=False, roofline=False))
    rep["default_ms_per_step"] = r["ms_per_step"]
    return rep


def fp4_from_bf16():
    """Four times the measured dense bf16 GEMM throughput of MEASURED_PEAKS.json
    (flop/s; the dense FP4 : BF16 rate ratio of B200), and its source."""
    try:
        bf16 = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"] * 1e12
        src = "4 x MEASURED_PEAKS.json bf16_tflops (cuBLAS bf16 burst)"
    except Exception:
        bf16, src = 1.59e15, "4 x the fallback bf16 1.59 PFLOP/s"
    return 4.0 * bf16, src


def traffic_from_profiles(kernel: str, name: str):
    """DRAM bytes per launch of `kernel` on this workload, measured by one ncu
    capture and recorded under profiles/ (None when that kernel was not
    captured on this workload)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        v = json.load(open(p)).get(kernel, {}).get(name)
        return float(v) if isinstance(v, (int, float)) else None
    except Exception:
        return None


# ------------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--popcount", action="store_true",
                    help="count DNA with the bit-plane popcount kernel instead of tensor cores")
    ap.add_argument("--mode", default="all",
                    choices=["all", "plain", "configs", "batched", "served", "bootstrap",
                             "njinit", "parse", "text"],
                    help="all: the plain workload line plus the other configurations and the "
                         "batched, served, bootstrap, parse, text and NJ set-up figures")
    ap.add_argument("--nj-n", type=int, default=10000,
                    help="sequences (and columns) of the NJ set-up workload (njinit)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    gen, n, L, type_, model = WORKLOADS[args.workload]
    config = {"workload": args.workload, "n": n, "L": L, "type": type_, "model": model,
              "kernel": ("popcount" if (args.popcount or (
                  type_ != "dna" and residue_ranks(make_alignment(args.workload)) > 31))
                  else "tcgen05"),
              "generator": gen, "seed": 0, "parallelism": f"tiles/{world}" if world > 1 else "single",
              "l2": "256 MiB buffer written between timed steps (L2 flushed)"}

    if args.impl == "reference":
        if rank != 0:
            return
        seqs = make_alignment(args.workload)
        # each step a bounded sample, the whole run a few minutes at most
        budget = max(0.5, min(8.0, 150.0 / max(1, args.warmup + args.steps)))
        cpu = cpu_reference(seqs, model, type_, args.warmup, args.steps, budget_s=budget)
        if cpu is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/ref_harness not built (needs the reference sources)"}))
            return
        line = {"impl": "reference", "metric": "pair-column comparisons/s", "value": cpu["value"],
                "unit": "pair-columns/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * sum(cpu["step_s"]) / len(cpu["step_s"]),
                "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "u32", "data": "synthetic", "config": config,
                "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": cpu["value"], "unit": "pair-columns/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    res = measure_workload(args.workload, args.steps, args.warmup, rank, world, local_rank,
                           popcount=args.popcount)
    if rank == 0:
        tc = res["kernel"] == "tcgen05"
        line = {"metric": "pair-column comparisons/s", "value": res["value"],
                "unit": "pair-columns/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "fp4" if tc else "u32",
                "dtype_note": ("exact integer counts: the FP4 e2m1 operands hold -1, 0, +1 "
                               "exactly and every f32 tensor sum is an integer below 2^24; the "
                               "transform is the reference's float/double arithmetic" if tc else
                               "exact integer counts from bit planes (POPC/LOP3)"),
                "data": "synthetic", "config": config, "roofline": res["roofline"],
                "e2e": res["e2e"], "clocks": res["clocks"], "stages_ms": res["stages_ms"],
                "gpu_launches": res["gpu_launches_per_step"] * args.steps}
        if world == 1:
            # the bucket's tuned launch choice (the headline) against the defaults
            try:
                line["tuning"] = tuning_report(args.workload, args.steps, local_rank,
                                               args.popcount, res["ms_per_step"])
            except Exception as e:  # noqa: BLE001
                line["tuning"] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
        if not args.no_cpu_baseline and world == 1:
            seqs = make_alignment(args.workload)
            cpu = cpu_reference(seqs, model, type_, 0, 1)
            line["cpu_baseline"] = ({k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
                                    if cpu else None)
        # The other single-GPU configurations of the workload list, each with its
        # own roofline, end-to-end figure and CPU baseline (guarded: a failure is
        # reported in the line, which is still printed).
        if args.mode in ("all", "configs") and world == 1:
            line["configs"] = {}
            for name in OTHER_CONFIGS:
                try:
                    r = measure_workload(name, min(args.steps, 10), 3, local_rank=local_rank,
                                         popcount=args.popcount)
                    r.pop("clocks", None)
                    if not args.no_cpu_baseline:
                        _, _, _, t_, m_ = WORKLOADS[name]
                        cpu = cpu_reference(make_alignment(name), m_, t_, 0, 1, budget_s=8.0)
                        r["cpu_baseline"] = ({k: cpu[k] for k in
                                              ("value", "unit", "cores", "kind", "sample")}
                                             if cpu else None)
                    line["configs"][name] = r
                except Exception as e:  # noqa: BLE001
                    line["configs"][name] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
        # the batched and served forms are single-GPU (replicas at N > 1); an
        # extra figure that fails is reported as such, the line still printed
        extras = (("batched", run_batched), ("served", run_served),
                  ("bootstrap", run_bootstrap), ("parse", run_parse), ("text", run_text),
                  ("nj_init", lambda a, r: run_nj_init(a, r, n=a.nj_n, L=a.nj_n)))
        modes = {"batched": "batched", "served": "served", "bootstrap": "bootstrap",
                 "parse": "parse", "text": "text", "nj_init": "njinit"}
        for key, fn in extras:
            if args.mode in ("all", modes[key]) and world == 1:
                try:
                    line[key] = fn(args, local_rank)
                except Exception as e:  # noqa: BLE001
                    line[key] = {"error": f"{type(e).__name__}: {str(e)[:300]}"}
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
