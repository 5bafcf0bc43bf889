"""The learned style selector (committed parameters) on graphs it was not
trained on (the held-out set of `selector.eval_specs()`, fixed before
training: RMAT / ER / grid of 2^18 and 2^20 vertices, seeds 7000-7005).

* It never changes a result.
* Against the frontier-size rule it falls back to (the heuristic), it is not
  slower overall: median of 7 resident traversals per case, BFS / SSSP / CC.
* Where the network overrides the rule (styles the rule never picks, such as
  the topology-driven pull on grids), it is faster: that is what the trained
  network adds to the method without it.
"""
import math

import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle
from indigo2suite_b200 import selector as S

pytestmark = pytest.mark.gpu

RULE_STYLES = {i2.VARIANTS.index(v) for v in ("vp_thread", "vp_cta", "pull_frontier", "union_find")}


@pytest.fixture(scope="module")
def params(gpu):
    p = np.fromfile(S.PARAMS_PATH, np.float32)
    assert p.size == i2.mlp_param_count()
    i2.mlp_set_params(p)
    return p


def _median_ms(dg, algo, src, variant, runs=7):
    dg.run_device(algo, src, variant=variant)
    return sorted(dg.run_device(algo, src, variant=variant).seconds for _ in range(runs))[runs // 2] * 1e3


def _geo(xs):
    return math.exp(sum(math.log(x) for x in xs) / len(xs))


def test_learned_results_are_bit_exact(params):
    for g in (i2.gen_rmat(16, 16, seed=901), i2.gen_grid(160, 0.05, 0.001, 902), i2.gen_er(30000, 120000, 903)):
        dg = i2.DeviceGraph.upload(g)
        src = int(np.argmax(g.degrees()))
        d, rep = dg.bfs(src, variant="learned")
        np.testing.assert_array_equal(d, oracle.bfs(g, src))
        assert sum(rep.variant_hist) == rep.iterations
        np.testing.assert_array_equal(dg.sssp(src, variant="learned")[0], oracle.sssp(g, src))
        np.testing.assert_array_equal(dg.cc(variant="learned")[0], oracle.cc(g))
        dg.free()


def test_learned_not_slower_than_rule_and_faster_where_it_overrides(params):
    ratios, overridden = [], []
    for spec in S.eval_specs():
        g = spec.build()
        dg = i2.DeviceGraph.upload(g)
        src = int(np.argmax(g.degrees()))
        for algo in (i2.I2_BFS, i2.I2_SSSP, i2.I2_CC):
            _, rep = dg._run(algo, src, "learned", i2.I2_LOOP_GRAPH, 0, False, None)
            r = _median_ms(dg, algo, src, "learned") / _median_ms(dg, algo, src, "heuristic")
            ratios.append(r)
            if any(n and k not in RULE_STYLES for k, n in enumerate(rep.variant_hist)):
                overridden.append(r)
        dg.free()
    assert _geo(ratios) <= 1.03, ratios
    assert len(overridden) >= 3, ratios
    assert _geo(overridden) < 1.0, overridden
