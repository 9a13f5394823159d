import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden_files():
    """The alignment fixtures (the NJ set-up fixtures nj_*.npz hold matrices)."""
    return sorted(p for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("nj_"))


def load_golden(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    d["names"] = bytes(d["names"]).decode().split("\n")
    d["fmt"] = bytes(d["fmt"]).decode()
    d["type_arg"] = bytes(d["type_arg"]).decode()
    d["name"] = os.path.basename(path)[:-4]
    return d


def golden_type(g):
    t = g["type_arg"]
    return int(g["ref_type"]) if t == "auto" else (0 if t == "d" else 1)


@pytest.fixture(scope="session")
def ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rapidnj_b200 import api
    c = api.Context(0)
    yield c
    c.close()
