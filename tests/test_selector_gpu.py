"""The learned style selector (committed parameters) on graphs it was not
trained on: it never changes a result, and on high-diameter graphs it is faster
than the fixed frontier-size heuristic it replaces."""
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


def test_learned_beats_the_fixed_heuristic_on_held_out_graphs(params):
    # What the trained network adds over the fixed rule: on high-diameter
    # graphs it moves BFS and SSSP iterations to the pull and topology styles,
    # where the rule keeps the push. On held-out 2^18-vertex grids (three
    # seeds, two B200 boxes) that measured 0.89-0.99x the rule's time; on
    # 2^20-vertex grids the two are at par (0.99-1.06x), and on RMAT/ER graphs
    # and for CC (both take union-find) they are at par too, so those cases
    # are only checked for not losing much.
    gains, par = [], []
    for spec in (S.GraphSpec("grid", 18, 8104), S.GraphSpec("grid", 18, 8106), S.GraphSpec("grid", 20, 8105)):
        g = spec.build()
        dg = i2.DeviceGraph.upload(g)
        src = int(np.argmax(g.degrees()))
        for algo in (i2.I2_BFS, i2.I2_SSSP):
            r = _median_ms(dg, algo, src, "learned", 7) / _median_ms(dg, algo, src, "heuristic", 7)
            (gains if spec.scale == 18 else par).append(r)
        dg.free()
    geo = math.exp(sum(math.log(r) for r in gains) / len(gains))
    assert geo < 0.98, gains
    assert max(par) < 1.15, par
