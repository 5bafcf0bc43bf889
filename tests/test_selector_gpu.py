"""The learned style selector (committed parameters) on graphs it was not
trained on: it never changes a result, and on high-diameter graphs it takes
the pull and topology styles that the fixed frontier-size heuristic never
picks there, without losing much time against it."""
import math

import numpy as np
import pytest

import indigo2suite_b200 as i2
import oracle
from indigo2suite_b200 import selector as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def params(gpu):
    p = np.fromfile(S.PARAMS_PATH, np.float32)
    assert p.size == i2.mlp_param_count()
    i2.mlp_set_params(p)
    return p


def _median_ms(dg, algo, src, variant, runs=5):
    dg.run_device(algo, src, variant=variant)
    return sorted(dg.run_device(algo, src, variant=variant).seconds for _ in range(runs))[runs // 2] * 1e3


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


def test_learned_moves_grid_iterations_to_pull_styles(params):
    # What the trained network adds over the fixed rule on high-diameter
    # graphs: it moves BFS and SSSP iterations from the push to the pull and
    # topology styles, which the rule never picks on grids. Its time against
    # the rule's on held-out grids of 2^18 and 2^20 vertices measured
    # 0.89-1.07x, depending on the box and the build (the push has become
    # faster since the network was trained), so of the time only "not much
    # slower" is asserted.
    pull = {i2.VARIANTS.index("pull_frontier"), i2.VARIANTS.index("pull_topo")}
    ratios = []
    for spec in (S.GraphSpec("grid", 18, 8104), S.GraphSpec("grid", 18, 8106), S.GraphSpec("grid", 20, 8105)):
        g = spec.build()
        dg = i2.DeviceGraph.upload(g)
        src = int(np.argmax(g.degrees()))
        for algo in (i2.I2_BFS, i2.I2_SSSP):
            _, rl = dg._run(algo, src, "learned", i2.I2_LOOP_GRAPH, 0, False, None, None)
            _, rh = dg._run(algo, src, "heuristic", i2.I2_LOOP_GRAPH, 0, False, None, None)
            assert sum(rl.variant_hist[k] for k in pull) > 0.2 * rl.iterations, (spec, algo, rl.variant_hist)
            assert sum(rh.variant_hist[k] for k in pull) == 0, (spec, algo, rh.variant_hist)
            ratios.append(_median_ms(dg, algo, src, "learned", 7) / _median_ms(dg, algo, src, "heuristic", 7))
        dg.free()
    geo = math.exp(sum(math.log(r) for r in ratios) / len(ratios))
    assert geo < 1.15, ratios
