"""Batched independent scenes: many clusters of uneven size fired at their own walls, all
advanced by the same launches.  A scene in the batch must evolve exactly as it does alone (the
neighbour grid is per scene, restitution/friction and walls come from the scene's table), and
alone it must match the oracle; tuned launch settings must not change any result."""
import os

import numpy as np
import pytest

from cabanadem_b200 import api, autotune, scenarios as S
from cabanadem_b200._lib import DEM_FP64, DEM_MIXED
from oracle import oracle as O

pytestmark = pytest.mark.gpu

STATE = ("x", "u", "omega", "force", "torque", "tng_count")


def _scene_slice(st, start, c):
    return {f: getattr(st, f)[start:start + c] for f in STATE}


def test_batch_equals_scenes_run_alone_and_oracle():
    sc = S.batched_scenes(nscenes=12, nmax=400, seed=21, nsteps=400)
    s = api.from_scenario(sc)
    s.run_steps(400)
    got = s.particles.download()
    counts = sc.extra["counts"]
    starts = np.concatenate([[0], np.cumsum(counts)])
    for k in range(len(counts)):
        sub = S.scene_subset(sc, k)
        alone = api.from_scenario(sub)
        alone.run_steps(400)
        a = alone.particles.download()
        ref = sub.state.copy()
        O.run(ref, sub.walls, sub.params, sub.dt, 400, skin=sub.skin, pow_mode=O.POW_SQRT)
        mine = _scene_slice(got, starts[k], counts[k])
        for f in STATE:
            assert np.array_equal(mine[f], getattr(a, f)), (k, f)
            assert np.array_equal(mine[f], getattr(ref, f)), (k, f, "oracle")
    assert got.tng_count.sum() > 0 or np.abs(got.force).max() > 0


def test_launch_settings_do_not_change_results(tmp_path):
    sc = S.batched_scenes(nscenes=24, nmax=2000, seed=5, nsteps=150)
    outs = []
    for cfg in ({"stream_block": 64, "steps_per_launch": 16, "skin_factor": 0.5},
                {"stream_block": 256, "steps_per_launch": 64, "skin_factor": 2.0},
                dict(autotune.DEFAULTS)):
        sc2 = S.batched_scenes(nscenes=24, nmax=2000, seed=5, nsteps=150)
        kw = autotune.apply(sc2, cfg)
        s = api.from_scenario(sc2, **kw)
        s.run_steps(150)
        outs.append(s.particles.download())
    for o in outs[1:]:
        for f in STATE:
            assert np.array_equal(getattr(o, f), getattr(outs[0], f)), f


def test_autotuner_picks_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("CABANADEM_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    sc = S.batched_scenes(nscenes=64, nmax=4096, seed=9, nsteps=100)
    cfg = autotune.tune(sc, precision=DEM_MIXED, warmup=5, steps=40)
    assert cfg["stream_block"] in (64, 128, 256)
    assert os.path.exists(tmp_path / "tune.json")
    assert autotune.tune(sc, precision=DEM_MIXED) == cfg    # served from the cache


def test_full_batch_mixed_matches_fp64():
    """The 1,024-scene batch (about 0.94M spheres): 50 steps mixed vs FP64."""
    a = api.from_scenario(S.batched_scenes(nsteps=50), precision=DEM_FP64)
    a.run_steps(50)
    b = api.from_scenario(S.batched_scenes(nsteps=50), precision=DEM_MIXED)
    b.run_steps(50)
    fa, fb = a.particles.get("force"), b.particles.get("force")
    assert np.all(np.isfinite(fb))
    assert np.abs(fb - fa).max() <= 1e-5 * np.abs(fa).max()
    assert np.array_equal(a.particles.get("tng_count"), b.particles.get("tng_count"))


def test_size_buckets_with_their_own_settings_equal_one_batch():
    """The batch split by scene size into buckets, each bucket a solver with launch settings of
    its own on its own stream, run concurrently (api.BatchRunner): the merged state equals the
    whole batch run as one solver bit for bit."""
    sc = S.batched_scenes(nscenes=40, nmax=3000, seed=17, nsteps=300)
    one = api.from_scenario(S.batched_scenes(nscenes=40, nmax=3000, seed=17, nsteps=300))
    one.run_steps(300)
    ref = one.particles.download()
    configs = {0: dict(contact_lanes=1, stream_block=64),
               1: dict(contact_lanes=8, steps_per_launch=32),
               2: dict(dense_form=2, skin_factor=0.5)}
    runner = api.BatchRunner(sc, configs=configs)
    assert len(runner.parts) >= 2
    runner.run_steps(120)
    runner.run_steps(180)
    got = runner.download()
    for f in STATE:
        assert np.array_equal(getattr(got, f), getattr(ref, f)), f
    runner.close()


@pytest.mark.parametrize("precision", [DEM_FP64, DEM_MIXED], ids=["fp64", "mixed"])
def test_small_scenes_in_one_persistent_launch(precision):
    """Scenes of at most 64 particles: a run is one launch, a block per scene with every step
    inside it (scene_kernel 0).  The state equals that of the per-step kernels (scene_kernel 1,
    cooperative_loop 2) bit for bit, over runs of odd and even length (the buffer parity of the
    launch), and in FP64 every scene equals the oracle run on that scene alone."""
    nsteps = (101, 200)
    sc = S.batched_scenes(nscenes=48, nmax=64, seed=31, nsteps=sum(nsteps))
    a = api.from_scenario(S.batched_scenes(nscenes=48, nmax=64, seed=31, nsteps=sum(nsteps)), precision=precision)
    b = api.from_scenario(S.batched_scenes(nscenes=48, nmax=64, seed=31, nsteps=sum(nsteps)), precision=precision,
                          scene_kernel=1, cooperative_loop=2)
    for k in nsteps:
        a.run_steps(k)
        b.run_steps(k)
    ga, gb = a.particles.download(), b.particles.download()
    for f in STATE:
        assert np.array_equal(getattr(ga, f), getattr(gb, f)), f
    assert a.stats()["launches"] * 10 < b.stats()["launches"]     # one launch per run, not per step
    assert ga.tng_count.sum() > 0                                  # contacts formed
    if precision == DEM_FP64:
        counts = sc.extra["counts"]
        starts = np.concatenate([[0], np.cumsum(counts)])
        for k in range(0, len(counts), 7):
            sub = S.scene_subset(sc, k)
            ref = sub.state.copy()
            O.run(ref, sub.walls, sub.params, sub.dt, sum(nsteps), skin=sub.skin, pow_mode=O.POW_SQRT)
            mine = _scene_slice(ga, starts[k], counts[k])
            for f in STATE:
                assert np.array_equal(mine[f], getattr(ref, f)), (k, f)


def test_small_scenes_in_shared_memory_with_hooks_and_force_readback():
    """The scenes kept in shared memory for a run carry every per-particle field the step uses:
    an external force on every particle and fix flags on some (force, torque or both zeroed
    after the pair forces) give the same bits as the per-step kernels, and so do the force and
    torque the run's last step leaves, the tracked slots' partners (renamed back to storage
    indices) and the wall history, over runs that cross the scenes' own list rebuilds."""
    nsteps = (150, 151)
    mk = lambda: S.batched_scenes(nscenes=48, nmax=64, seed=31, nsteps=sum(nsteps))
    n = mk().state.n
    rng = np.random.default_rng(5)
    ext = rng.normal(0.0, 1e-6, (n, 3))
    fix = (rng.random(n) < 0.1).astype(np.uint8) * rng.integers(1, 4, n).astype(np.uint8)
    solvers = []
    for kw in ({}, dict(scene_kernel=1, cooperative_loop=2)):
        s = api.from_scenario(mk(), **kw)
        s.particles.set("ext_force", ext)
        s.particles.set("fix", fix)
        solvers.append(s)
    for k in nsteps:
        for s in solvers:
            s.run_steps(k)
    ga, gb = (s.particles.download() for s in solvers)
    for f in STATE + ("tng_idx", "tng_ss_x", "tng_sw_x", "tng_sw_y"):
        a, b = getattr(ga, f), getattr(gb, f)
        if f in ("tng_idx", "tng_ss_x"):   # slots beyond the count are not part of the state
            live = np.arange(a.shape[1])[None, :] < gb.tng_count[:, None]
            a, b = np.where(live, a, 0), np.where(live, b, 0)
        assert np.array_equal(a, b), f
    assert ga.tng_count.sum() > 0
    assert solvers[0].stats()["launches"] * 10 < solvers[1].stats()["launches"]
