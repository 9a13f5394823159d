"""rnj_write_matrix_text_device: the "-o m" text of a device matrix formatted on
the device must be byte-identical to the host writer's (snprintf "%.6f "), which
the reference's own "-o m" output pins (tests/test_oracle_golden.py,
tests/test_gpu_dropin.py)."""
import numpy as np
import pytest

from rapidnj_b200 import api

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def both(ctx, tmp_path, m, names, pad=0):
    n = m.shape[0]
    host = tmp_path / "h.txt"
    dev = tmp_path / "d.txt"
    api.write_matrix_text(str(host), names, m)
    buf = torch.zeros((n, n + pad), dtype=torch.float32, device="cuda")
    buf[:, :n] = torch.from_numpy(np.ascontiguousarray(m, dtype=np.float32)).cuda()
    api.write_matrix_text_device(ctx, str(dev), names, buf[:, :n])
    a, b = host.read_bytes(), dev.read_bytes()
    if a != b:
        k = next(i for i in range(min(len(a), len(b))) if a[i] != b[i])
        raise AssertionError(f"first difference at byte {k}: {a[k-40:k+40]!r} vs {b[k-40:k+40]!r}")
    return a


def matrix(n, seed):
    rng = np.random.default_rng(seed)
    m = (rng.random((n, n)) * 3.0).astype(np.float32)
    flat = m.reshape(-1)
    k = flat.size
    idx = rng.integers(0, k, size=(6, max(1, k // 50)))
    flat[idx[0]] = -0.0
    flat[idx[1]] = (rng.integers(-4000, 4000, idx.shape[1]) / 128.0).astype(np.float32)  # ties
    flat[idx[2]] = (rng.random(idx.shape[1]) * 7.9e9).astype(np.float32)
    flat[idx[3]] = -(rng.random(idx.shape[1]) * 1e-6).astype(np.float32)  # "-0.000000"
    flat[idx[4]] = (rng.random(idx.shape[1]) * 1e-6).astype(np.float32)
    flat[idx[5]] = 0.0
    return m


@pytest.mark.parametrize("n", [1, 2, 33, 700, 3000])
def test_identical_to_host_writer(ctx, tmp_path, n):
    names = [("seq_%d" % i) * (1 + i % 3) for i in range(n)]
    both(ctx, tmp_path, matrix(n, n), names, pad=n % 3)


def test_rows_printed_by_the_host(ctx, tmp_path):
    m = matrix(300, 7)
    m[3, 5] = np.inf
    m[10, 0] = -np.inf
    m[20, 7] = np.nan
    m[40, 40] = 1e10
    m[41, 2] = -3e12
    m[42, 9] = 8e9
    both(ctx, tmp_path, m, [f"r{i}" for i in range(300)])


def test_empty_names_and_large_file(ctx, tmp_path):
    # more than one 64 MB band, names of every length including empty
    n = 3100
    m = matrix(n, 11)
    names = ["" if i % 17 == 0 else "x" * (i % 40) for i in range(n)]
    text = both(ctx, tmp_path, m, names)
    assert len(text) > (64 << 20)


def test_distance_matrix_text(ctx, tmp_path):
    from rapidnj_b200 import synth
    s = synth.tree_dna(800, 900, seed=3)
    s[5] = s[6]  # an identical pair: K2P gives -0 between them
    aln = ctx.alignment(s, 0)
    out = torch.empty((800, 800), dtype=torch.float32, device="cuda")
    ctx.distance_into(aln, "kim", out)
    aln.close()
    text = both(ctx, tmp_path, out.cpu().numpy(), [f"s{i}" for i in range(800)])
    assert b"-0.000000" in text
