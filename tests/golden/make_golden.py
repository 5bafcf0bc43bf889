"""Generate tests/golden/golden.npz from the reference's own code.

Run where the reference tree is present (it is not on GPU machines):

    python tests/golden/make_golden.py

Contents, per case:
* the CSR (nindex, nlist, eweight) of the reference's 7 small inputs
  (small-inputs/*.egr) and of three small seeded synthetic graphs;
* BFS levels and SSSP distances from the reference's CPUserialDijkstra
  (include/bfs_vertex_omp.h, include/sssp_edge_omp.h, compiled unchanged by
  oracle/Makefile), from every source of the small inputs and from source 0 of
  the synthetic graphs; small inputs have no weights, so SSSP uses the
  reference's synthetic weights computed by its own harness formula;
* CC labels (minimum vertex ID per component), accepted by the reference's own
  CC verifier (include/cc_vertex_omp.h main(), via oracle/_ref/inject_cc_vertex).
"""
from __future__ import annotations

import os
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import indigo2suite_b200 as i2  # noqa: E402
import oracle  # noqa: E402

# the reference tree: $I2_REFERENCE_ROOT (the same variable oracle/Makefile reads)
SMALL = Path(os.environ.get("I2_REFERENCE_ROOT", "/root/reference")) / "small-inputs"


def add_case(out: dict, name: str, g: i2.ECLGraph, sources: list[int]) -> None:
    if g.eweight is None:
        g = i2.synth_weights(g)
    out[f"{name}/nindex"] = g.nindex
    out[f"{name}/nlist"] = g.nlist
    out[f"{name}/eweight"] = g.eweight
    out[f"{name}/sources"] = np.array(sources, np.int32)
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "g.egr")
        oracle.write_egr(g, p)
        for s in sources:
            b = oracle.ref_serial("bfs", g, s)
            d = oracle.ref_serial("sssp_edge", g, s)
            ok1, _ = oracle.ref_verify("bfs_vertex", p, b, s)
            ok2, _ = oracle.ref_verify("sssp_edge", p, d, s)
            assert ok1 and ok2, name
            out[f"{name}/bfs/{s}"] = b
            out[f"{name}/sssp/{s}"] = d
        lab = oracle.cc(g)
        ok, _ = oracle.ref_verify("cc_vertex", p, lab, None)
        assert ok, name
        out[f"{name}/cc"] = lab


def main() -> None:
    oracle.build(ref=True)
    out: dict[str, np.ndarray] = {}
    names = []
    for f in sorted(SMALL.glob("*.egr")):
        g = i2.read_eclgraph(str(f))
        name = "small_" + f.stem
        add_case(out, name, g, list(range(g.nodes)))
        names.append(name)
    for name, g in [("er_n1000_m4000_s7", i2.gen_er(1000, 4000, 7)),
                    ("rmat_s10_ef16_s3", i2.gen_rmat(10, 16, seed=3)),
                    ("grid_32_s5", i2.gen_grid(32, 0.05, 0.01, 5))]:
        add_case(out, name, g, [0])
        names.append(name)
    out["cases"] = np.array(names)
    np.savez_compressed(Path(__file__).with_name("golden.npz"), **out)
    print(f"wrote {len(names)} cases")


if __name__ == "__main__":
    main()
