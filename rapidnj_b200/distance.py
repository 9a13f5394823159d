"""The reference's distance-calculator interface, backed by the sm_100a path.

Mirrors, name for name, the classes rapidNJ's driver uses (src/main.cpp:237-286):

* ``Dataloader``      -- dataloader.hpp:13-101 (readData, getSequenceCount,
                         getSequenceLength, getSequenceNames, getSequences, type,
                         fastdist); FASTA / Stockholm parsing with the reference
                         rules happens in librnjgpu.so (rnj_msa_read).
* ``JCdistance``      -- JCdistance.hpp:11-35: JCdistance(verbose, fastdist,
                         loader, dm); computeDistanceMatrix(numThreads);
                         getDistanceMatrix().
* ``KimuraDistance``  -- KimuraDistance.hpp:9-39: KimuraDistance(verbose,
                         fastdist, loader, dm); computeDistances(numThreads);
                         getDistanceMatrix().

``getDistanceMatrix()`` returns the full post-processed float32 matrix (rows
are what the reference's ``distType**`` holds).  ``numThreads`` sizes only the
host copy-out; the pairs are computed on the GPU.  With ``dm`` (a
``DiskRows``-like object with ``writeArray(row, i, n)``) the rows are streamed
to it instead, as the reference's disk-matrix mode does.
"""
from __future__ import annotations

import sys

import numpy as np

from . import api
from ._native import RNJ_DNA, RNJ_PROTEIN, RNJ_UNKNOWN, RnjError

DNA, PROTEIN, UNKNOWN = RNJ_DNA, RNJ_PROTEIN, RNJ_UNKNOWN

_default_ctx = None


def default_context() -> api.Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = api.Context(0)
    return _default_ctx


class Dataloader:
    """Alignment loader with the reference's accessors (dataloader.hpp:20-27, 84-86)."""

    def __init__(self, fmt: str | None = None):
        self.fmt = fmt
        self.type = UNKNOWN
        self.fastdist = True
        self.names: list[str] = []
        self.chars = np.zeros((0, 0), np.uint8)

    def readData(self, filename: str, fastdist: bool, verbose: bool, type_: int = UNKNOWN,
                 gpu: bool = False) -> None:
        names, chars, detected = api.read_alignment(filename, self.fmt)
        self.fastdist = fastdist
        self.type = detected if type_ == UNKNOWN else type_
        self.names, self.chars = names, chars
        if chars.shape[0] <= 1:
            raise RnjError(5, f"Found {chars.shape[0]} sequences in the input file. At least 2 "
                              "sequences are needed to build a tree.")
        if verbose:
            print(f"Input type determined as {'DNA' if self.type == DNA else 'PROTEIN'}.",
                  file=sys.stderr)
            print(f"Number of sequences: {chars.shape[0]}", file=sys.stderr)
            print(f"Sequence length: {chars.shape[1]}", file=sys.stderr)

    @classmethod
    def from_array(cls, chars: np.ndarray, type_: int = UNKNOWN, fastdist: bool = True,
                   names=None) -> "Dataloader":
        d = cls()
        d.chars = np.ascontiguousarray(chars, dtype=np.uint8)
        d.fastdist = fastdist
        d.type = api.detect_type(d.chars[0].tobytes()) if type_ == UNKNOWN else type_
        d.names = list(names) if names is not None else [f"s{i}" for i in range(d.chars.shape[0])]
        return d

    def getSequenceCount(self) -> int:
        return int(self.chars.shape[0])

    def getSequenceLength(self) -> int:
        return int(self.chars.shape[1])

    def getSequenceNames(self) -> list[str]:
        return self.names

    def getSequences(self) -> np.ndarray:
        return self.chars


class _DistanceBase:
    MODEL = "kim"

    def __init__(self, verbose: bool, fastdist: bool, loader: Dataloader, dm=None,
                 ctx: api.Context | None = None, compat_wrap: bool = False):
        self.verbose = verbose
        self.fastdist = fastdist
        self.loader = loader
        self.dm = dm
        self.ctx = ctx or default_context()
        self.compat_wrap = compat_wrap
        self.seqCount = loader.getSequenceCount()
        self.maxDistance = 0.0
        self._matrix = None

    def _compute(self, numThreads: int) -> None:
        full = self.dm is not None
        aln = self.ctx.alignment(self.loader.getSequences(), self.loader.type, self.fastdist,
                                 self.compat_wrap, full_rows=full)
        try:
            mat = self.ctx.distance(aln, self.MODEL)
        finally:
            aln.close()
        try:
            self.maxDistance = mat.max
            if self.dm is None:
                self._matrix = mat.to_numpy(numThreads)
            else:
                n = self.seqCount
                row = np.empty(n, np.float32)
                for i in range(n):
                    mat.copy_rows([row], i, numThreads)
                    self.dm.writeArray(row, i, n)
        finally:
            mat.close()

    def getDistanceMatrix(self):
        return self._matrix


class JCdistance(_DistanceBase):
    MODEL = "jc"

    def computeDistanceMatrix(self, numThreads: int) -> None:
        self._compute(numThreads)


class KimuraDistance(_DistanceBase):
    MODEL = "kim"

    def computeDistances(self, numThreads: int) -> None:
        self._compute(numThreads)
