"""The autotuner's host logic on CPU, with a synthetic cost in place of the timed device runs:
the coordinate search from the defaults finds the best setting of each knob in turn, the
result is cached per size bucket (log2 n, precision, batched or single) and a cached bucket is
answered without timing anything; apply() turns a configuration into the scenario's skin and
the solver's keyword arguments."""
import json

from cabanadem_b200 import autotune, scenarios as S


def _cost(cfg):
    # separable, minimum at contact_lanes 4, dense_form 2, stream_split 1, stream_block 256,
    # steps_per_launch 32, skin_factor 0.5
    return ({0: 4.0, 1: 3.0, 4: 1.0, 8: 2.0}[cfg["contact_lanes"]] + {0: 3.0, 1: 2.0, 2: 1.0}[cfg["dense_form"]]
            + {0: 2.0, 1: 1.0}[cfg["stream_split"]]
            + {64: 3.0, 128: 2.0, 256: 1.0}[cfg["stream_block"]] + {0: 2.0, 32: 1.0}[cfg["steps_per_launch"]]
            + {0.5: 1.0, 1.0: 2.0, 2.0: 3.0, 4.0: 4.0}[cfg["skin_factor"]])


BEST = dict(contact_lanes=4, dense_form=2, stream_split=1, stream_block=256, steps_per_launch=32, skin_factor=0.5)
NTRIALS = 1 + 3 + 2 + 1 + 2 + 1 + 3     # defaults + every other candidate of each knob


def test_coordinate_search_and_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("CABANADEM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    calls = []

    def fake(sc, cfg, precision, warmup, steps, ctx=None):
        calls.append(dict(cfg))
        return _cost(cfg)
    monkeypatch.setattr(autotune, "time_config", fake)
    sc = S.random_box(n=300)
    cfg = autotune.tune(sc, precision=0)
    assert cfg == BEST
    assert calls[0] == autotune.DEFAULTS and len(calls) == NTRIALS
    table = json.loads((tmp_path / "tune.json").read_text())
    key = autotune.bucket(sc, 0)
    assert key == "n2^8|p0|single" and table[key]["config"] == cfg and table[key]["s_per_step"] == 6.0
    calls.clear()
    assert autotune.tune(S.random_box(n=400), precision=0) == cfg and calls == []   # same bucket: cached
    autotune.tune(sc, precision=1)
    assert len(calls) == NTRIALS                                      # another precision: tuned anew
    sc_skin = sc.skin
    kw = autotune.apply(sc, cfg)
    assert kw == dict(stream_block=256, steps_per_launch=32, contact_lanes=4, dense_form=2, stream_split=1)
    assert sc.skin == sc_skin * 0.5


def test_batched_bucket_is_separate():
    sc = S.batched_scenes(nscenes=8, nmax=64)
    assert "|p1|batched|scenes" in autotune.bucket(sc, 1)


def test_scene_size_buckets_split_and_key_the_tuning():
    """split_scenes groups a batch by scene size ([2, 64), [64, 1024), [1024, 8192]): every
    particle lands in exactly one bucket with its scene's wall and parameters, scenes keep their
    order, and each bucket has a tuning key of its own."""
    import numpy as np
    sc = S.batched_scenes(nscenes=60, nmax=3000, seed=4)
    parts = S.split_scenes(sc)
    assert [b for b, _, _ in parts] == sorted(b for b, _, _ in parts)
    rows = np.concatenate([sub.extra["rows"] for _, sub, _ in parts])
    assert np.array_equal(np.sort(rows), np.arange(sc.state.n))
    keys = {}
    for b, sub, ids in parts:
        counts = sc.extra["counts"][ids]
        assert all(S.scene_bucket_of(int(c)) == b for c in counts)
        assert np.array_equal(sub.state.x, sc.state.x[sub.extra["rows"]])
        assert [sub.extra["scene_params"][k] for k in range(len(ids))] == [sc.extra["scene_params"][k] for k in ids]
        assert np.array_equal(sub.walls.normal, sc.walls.normal[ids])
        keys[b] = autotune.bucket(sub, 1)
    assert len(set(keys.values())) == len(parts)
    assert all(k.endswith("|scenes%d" % b) for b, k in keys.items())


def test_packaged_b200_settings_cover_the_batch_buckets():
    """The launch settings shipped for B200 (used by BatchRunner when neither configurations nor
    tuning are given) cover every size bucket of the 1,024-scene batch, and every value is one
    the tuner could have kept (a default or a candidate)."""
    from cabanadem_b200._lib import DEM_MIXED
    sc = S.batched_scenes(seed=3)
    parts = S.split_scenes(sc)
    assert len(parts) == 3
    for b, sub, ids in parts:
        cfg = autotune.packaged(sub, DEM_MIXED)
        assert cfg is not None, autotune.bucket(sub, DEM_MIXED)
        assert set(cfg) == set(autotune.DEFAULTS)
        assert all(cfg[k] in autotune.CANDIDATES[k] or cfg[k] == autotune.DEFAULTS[k] for k in cfg)
    assert autotune.packaged(S.random_box(n=300), 0) is None
