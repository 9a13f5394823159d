"""Builds the launch-parameter table the library ships (tune_b200.txt beside
librnjgpu.so) by running the autotuner, rnj_tune, on this machine's GPU for
every bucket the standard workloads touch:

* the plain workloads: DNA 10,000 x 10,000, 50,000 x 1,000 and 512 x 2,000;
  protein 5,000 x 1,500;
* the batched mix (N in [32, 2048], L in [300, 5000]) and the served stream
  (N in [16, 4096], L in [200, 8000]): every (floor(log2 N), floor(log2 L))
  bucket of those ranges, DNA and protein, tuned at the geometric middle of the
  bucket clipped to the range.

A bucket is (alphabet, counting rules, floor(log2 N), floor(log2 L)); every
choice in it gives the same distances, only the time differs.  Usage:

    python -m rapidnj_b200.make_tune_table [--out PATH] [--device N]

The library reads the table at its first tuning lookup unless the environment
variable RNJ_TUNE_CACHE names another file.
"""
import argparse
import math
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))

PLAIN = [(10000, 10000, "dna"), (50000, 1000, "dna"), (512, 2000, "dna"), (5000, 1500, "protein")]
RANGES = [((32, 2048), (300, 5000)), ((16, 4096), (200, 8000))]  # batched, served


def bucket_shapes():
    """(n, L, alphabet) representatives of every bucket of the standard workloads."""
    seen, out = set(), []

    def add(n, L, t):
        key = (t, int(math.floor(math.log2(n))), int(math.floor(math.log2(L))))
        if key not in seen:
            seen.add(key)
            out.append((n, L, t))

    for n, L, t in PLAIN:
        add(n, L, t)
    for (n0, n1), (l0, l1) in RANGES:
        for kn in range(int(math.log2(n0)), int(math.log2(n1)) + 1):
            for kl in range(int(math.log2(l0)), int(math.log2(l1)) + 1):
                n = min(max(int(round(2 ** (kn + 0.5))), n0), n1)
                L = min(max(int(round(2 ** (kl + 0.5))), l0), l1)
                if n < 2 or int(math.log2(n)) != kn or int(math.log2(L)) != kl:
                    continue
                for t in ("dna", "protein"):
                    add(n, L, t)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=os.path.join(HERE, "tune_b200.txt"))
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    sys.path.insert(0, os.path.dirname(HERE))
    from rapidnj_b200 import api

    api.tune_clear()
    ctx = api.Context(args.device)
    shapes = bucket_shapes()
    t0 = time.time()
    for k, (n, L, t) in enumerate(shapes):
        p = ctx.tune(n, L, t)
        print(f"[{k + 1}/{len(shapes)}] {t} {n} x {L}: {p.as_dict()}", flush=True)
    api.tune_save(args.out)
    ctx.close()
    print(f"{len(shapes)} buckets in {time.time() - t0:.1f} s -> {args.out}")


if __name__ == "__main__":
    main()
