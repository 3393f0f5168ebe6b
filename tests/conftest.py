"""Shared test setup: the `gpu` marker, import paths, and small generators."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the cuda backend")


ALL_MODES = (0, 1, 2, 3, 4)  # SW, NW, HW, OV, SHW


def identity_matrix(al, m, x):
    """tests/common/mod.rs:13-20."""
    v = [x] * (al * al)
    for i in range(al):
        v[i * al + i] = m
    return v


DNA = identity_matrix(4, 2, -1)  # tests/common/mod.rs:23-25: +2/-1, go 2, ge 1


def all_sequences(alphabet, max_len):
    """tests/common/mod.rs:28-45: every sequence of length 0..=max_len."""
    out = [[]]
    frontier = [[]]
    for _ in range(max_len):
        nxt = [s + [a] for s in frontier for a in range(alphabet)]
        out.extend(nxt)
        frontier = nxt
    return out


class Lcg:
    """The deterministic PRNG of tests/sweeps.rs:23-28."""

    def __init__(self, seed):
        self.s = seed & (2**64 - 1)

    def next(self):
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & (2**64 - 1)
        return self.s >> 33

    def seq(self, length, al):
        return [self.next() % al for _ in range(length)]


def parse_fasta(path):
    """tests/common/mod.rs:197-218 (A,C,G,T,N -> 0..4)."""
    code = {"A": 0, "C": 1, "G": 2, "T": 3, "N": 4}
    recs, name, seq = [], None, []
    for line in open(path):
        line = line.strip()
        if line.startswith(">"):
            if name is not None:
                recs.append((name, seq))
            name, seq = line[1:].split()[0], []
        elif line:
            seq.extend(code[c] for c in line.upper())
    if name is not None:
        recs.append((name, seq))
    return recs


DATA = os.path.join(ROOT, "tests", "data")
