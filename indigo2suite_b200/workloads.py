"""Seeded synthetic workloads of the benchmark configurations.

* batch512: 512 graphs, vertex counts log-uniform in [1e3, 1e6], family drawn
  uniformly from ER (average degree 8), RMAT (edge factor 16, a=0.57 b=0.19
  c=0.19 on ceil(log2 n) bits, endpoints >= n rejected) and 2-D grid (side
  ceil(sqrt n), 5% of edges removed, 0.1% long-range edges added); int32
  weights uniform in [1, 255]; source = highest-degree vertex of each graph.
* grid4096: 4096 x 4096 grid, 5% of edges removed, 0.1% long-range edges.
* rmat(scale): RMAT, edge factor 16, a=0.57 b=0.19 c=0.19 d=0.05.

All graphs are symmetrised, deduplicated and free of self-loops; the seeds
make every run identical.
"""
from __future__ import annotations

import math

import numpy as np

from . import DeviceGraph, gen_er, gen_grid, gen_rmat_n


def batch_specs(count: int = 512, seed: int = 4, nmin: float = 1e3, nmax: float = 1e6):
    rng = np.random.default_rng(seed)
    specs = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        fam = ("er", "rmat", "grid")[int(rng.integers(0, 3))]
        specs.append((fam, n, int(rng.integers(1, 2**31 - 1))))
    return specs


def build(spec):
    fam, n, seed = spec
    if fam == "er":
        return gen_er(n, 4 * n, seed)
    if fam == "rmat":
        return gen_rmat_n(n, 16, 0.57, 0.19, 0.19, seed=seed)
    side = int(math.ceil(math.sqrt(n)))
    return gen_grid(side, 0.05, 0.001, seed=seed)


def build_device(spec) -> DeviceGraph:
    """The same graph as build(spec), generated on the device."""
    fam, n, seed = spec
    if fam == "er":
        return DeviceGraph.generate_er(n, 4 * n, seed)
    if fam == "rmat":
        return DeviceGraph.generate_rmat_n(n, 16, 0.57, 0.19, 0.19, seed=seed)
    side = int(math.ceil(math.sqrt(n)))
    return DeviceGraph.generate_grid(side, 0.05, 0.001, seed=seed)


def source(g) -> int:
    return int(np.argmax(np.diff(g.nindex.astype(np.int64))))
