"""Stage-kernel autotuners: nsf_autotune (one grid shape, single-grid kernel) and the ensemble's tile choice
(throwaway ensembles of the same members timed with each tile shape). Both cache their result as one JSON
line per key; a cached key is not timed again, and the tile a cache names is the one used."""
import json

import pytest

import nsfsi


def lines(path):
    with open(path) as f:
        return [json.loads(x) for x in f if x.strip()]


@pytest.mark.gpu
def test_autotune_caches_per_grid_shape(tmp_path):
    cache = str(tmp_path / "tiles.jsonl")
    cfg = nsfsi.ensemble_configs(n=1, steps=10)[0]
    tile, ns = nsfsi.autotune(cfg, cache=cache)
    assert tile in (0, 1) and (ns > 0).all()
    assert tile == (1 if ns[1] < ns[0] else 0)
    got = lines(cache)
    assert len(got) == 1 and got[0]["key"].endswith("/%dx%dx%d" % (cfg.NI, cfg.NJ, cfg.NK))
    assert got[0]["tile"] == tile
    tile2, ns2 = nsfsi.autotune(cfg, cache=cache)  # read back, not timed again
    assert tile2 == tile and list(ns2) == pytest.approx(list(ns), rel=1e-5)
    assert len(lines(cache)) == 1


@pytest.mark.gpu
def test_ensemble_tile_tuned_once_per_composition(tmp_path):
    cache = str(tmp_path / "tiles.jsonl")
    cfgs = nsfsi.ensemble_configs(n=5, steps=10)
    with nsfsi.Ensemble(cfgs, tune_cache=cache) as ens:
        tile, _, _ = ens.info()
        ens.march(2)
        ens.sync()
    got = lines(cache)
    assert len(got) == 1 and "/ensemble/" in got[0]["key"]
    assert got[0]["tile"] == tile == (1 if got[0]["ns_per_node"][1] < got[0]["ns_per_node"][0] else 0)
    # the same composition in another order: the cached choice, no new timing
    with nsfsi.Ensemble(cfgs[::-1], tune_cache=cache) as ens:
        assert ens.info()[0] == tile
    assert len(lines(cache)) == 1
    # a cache entry decides the tile shape
    forced = dict(got[0], tile=1 - tile)
    with open(cache, "w") as f:
        f.write(json.dumps(forced) + "\n")
    with nsfsi.Ensemble(cfgs, tune_cache=cache) as ens:
        assert ens.info()[0] == 1 - tile
        ens.march(2)
        ens.sync()
