"""Launch-shape knobs change only the speed of the step kernels, never the
numbers: every cell runs the same arithmetic however the grid is tiled and
however many time steps a launch fuses."""

from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

SETTINGS = [dict(ctas_per_sm=1, batch_tiles_per_cta=1, xchunk=0, tile_shape=0),
            dict(ctas_per_sm=2, batch_tiles_per_cta=16, xchunk=0, tile_shape=1),
            dict(ctas_per_sm=1, batch_tiles_per_cta=8, xchunk=5, tile_shape=2),
            dict(ctas_per_sm=2, batch_tiles_per_cta=8, xchunk=64, tile_shape=2),
            dict(ctas_per_sm=2, batch_tiles_per_cta=4, xchunk=0, tile_shape=1),
            dict(ctas_per_sm=2, batch_tiles_per_cta=8, xchunk=0, tile_shape=0, steps_per_pass=1),
            dict(ctas_per_sm=2, batch_tiles_per_cta=8, xchunk=0, tile_shape=0, steps_per_pass=2)]


def _problems():
    from shearwave_b200 import workloads as W

    return [W.problem_inclusions(s, n, seed=i, cfl=0.2)
            for i, (s, n) in enumerate([((40, 36, 50), 30), ((70, 21, 33), 25),
                                        ((18, 66, 130), 40)])]


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_knobs_do_not_change_results(cuda, precision):
    import shearwave_b200 as sw
    from shearwave_b200 import tune

    probs = _problems()
    keys = ("bx", "by", "bz", "rho", "mu", "dX", "dY", "dZ", "dT", "n_steps")
    ref = None
    for s in SETTINGS:
        with tune.knobs(**s):
            single = sw.shear_fdtd(**{k: probs[2][k] for k in keys},
                                   opts=dict(probs[2]["opts"], precision=precision))
            batch = sw.shear_fdtd_batch(probs, precision=precision)
        out = [single] + batch
        if ref is None:
            ref = out
            continue
        for a, b in zip(out, ref):
            for x, y in zip(a, b):
                assert (x == y).all(), s


def test_autotune_picks_a_candidate(cuda, tmp_path):
    from shearwave_b200 import tune

    probs = _problems()
    old = tune.get_knobs()
    try:
        cands = SETTINGS[:2]
        r = tune.autotune(probs, steps=10, repeats=1, candidates=cands,
                          cache=tmp_path / "t.json")
        assert r["best"] in cands and len(r["results"]) == 2
        assert all(x["gcell_steps_per_s"] > 0 for x in r["results"])
        assert tune.get_knobs() == {**old, **r["best"]}
        tune.set_knobs(**old)
        assert tune.apply_cached(probs, cache=tmp_path / "t.json") == r["best"]
    finally:
        tune.set_knobs(**old)
