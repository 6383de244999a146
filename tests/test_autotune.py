"""The autotuner's host logic on CPU, with a synthetic cost in place of the timed device runs:
the coordinate search from the defaults finds the best setting of each knob in turn, the
result is cached per size bucket (log2 n, precision, batched or single) and a cached bucket is
answered without timing anything; apply() turns a configuration into the scenario's skin and
the solver's keyword arguments."""
import json

from cabanadem_b200 import autotune, scenarios as S


def _cost(cfg):
    # separable, minimum at stream_block 256, steps_per_launch 64, skin_factor 0.5
    return ({64: 3.0, 128: 2.0, 256: 1.0}[cfg["stream_block"]] + {16: 3.0, 32: 2.0, 64: 1.0}[cfg["steps_per_launch"]]
            + {0.5: 1.0, 1.0: 2.0, 2.0: 3.0}[cfg["skin_factor"]])


def test_coordinate_search_and_cache(tmp_path, monkeypatch):
    monkeypatch.setenv("CABANADEM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    calls = []

    def fake(sc, cfg, precision, warmup, steps, ctx=None):
        calls.append(dict(cfg))
        return _cost(cfg)
    monkeypatch.setattr(autotune, "time_config", fake)
    sc = S.random_box(n=300)
    cfg = autotune.tune(sc, precision=0)
    assert cfg == dict(stream_block=256, steps_per_launch=64, skin_factor=0.5)
    assert calls[0] == autotune.DEFAULTS and len(calls) == 7          # defaults + 2 per knob
    table = json.loads((tmp_path / "tune.json").read_text())
    key = autotune.bucket(sc, 0)
    assert key == "n2^8|p0|single" and table[key]["config"] == cfg and table[key]["s_per_step"] == 3.0
    calls.clear()
    assert autotune.tune(S.random_box(n=400), precision=0) == cfg and calls == []   # same bucket: cached
    autotune.tune(sc, precision=1)
    assert len(calls) == 7                                            # another precision: tuned anew
    sc_skin = sc.skin
    kw = autotune.apply(sc, cfg)
    assert kw == dict(stream_block=256, steps_per_launch=64) and sc.skin == sc_skin * 0.5


def test_batched_bucket_is_separate():
    sc = S.batched_scenes(nscenes=8, nmax=64)
    assert autotune.bucket(sc, 1).endswith("|p1|batched")
