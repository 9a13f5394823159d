"""rapidnj_b200 -- rapidNJ's all-pairs distance estimation on B200 (sm_100a).

The product is the native library ``librnjgpu.so`` (C ABI in ``include/rnj.h``);
this package is its Python face:

* ``api``       contexts, packed alignments, device matrices, file reading
* ``distance``  the reference's ``JCdistance`` / ``KimuraDistance`` / loader interface
* ``synth``     seeded synthetic alignments of the benchmark workloads
"""
from . import api, distance, synth  # noqa: F401
from ._native import (RNJ_DNA, RNJ_FASTDIST, RNJ_JC, RNJ_KIMURA, RNJ_PROTEIN,  # noqa: F401
                      RNJ_UNKNOWN, RnjError)
from .api import Context, read_alignment, write_matrix_text  # noqa: F401
from .distance import Dataloader, JCdistance, KimuraDistance  # noqa: F401

__all__ = ["api", "distance", "synth", "Context", "Dataloader", "JCdistance", "KimuraDistance",
           "RnjError", "read_alignment", "write_matrix_text"]
