"""The learned surrogate on worlds: training on plain rollouts, the learned
step, and the judge / fallback runner.

* Training lowers the held-out one-step error (a scene never trained on, at
  a time inside the trained part of the rollout: after the first 20 steps of
  the lattice start, which only fit the normalisation) well below that of the
  method without the network (predicting the mean acceleration and density
  rate, i.e. the network's output zeroed) and below the untrained network.
* With a bound nothing can meet, every window falls back, and the run is bit
  for bit the plain run; with a bound nothing can exceed, no window does.
"""
import numpy as np
import pytest

import physics_engine_rs as pe
from helpers import assert_bits_equal, dam_break_params_pe
from physics_engine_rs import scenes
from physics_engine_rs import surrogate as S

pytestmark = pytest.mark.gpu

DT = 1e-4


def _world(seed, tanks=4):
    t, _ = scenes.batch_dam_break(tanks, seed, 2000, 3000, 0.3, 0.4)
    return pe.WcsphWorld.from_tanks(dam_break_params_pe(), t)


def _heldout_loss(sur, world, steps_before=150):
    world.run(DT, steps_before)
    a, b = S.tank_range(world, 0)
    sur.graph_from_world(world, a, b)
    world.step(DT)
    sur.targets_from_world(world, DT, update_stats=False)
    return sur.train_step(0.0)


def test_training_beats_the_method_without_the_network():
    train = _world(21)
    sur = S.Surrogate(seed=5)
    losses = S.train_on_rollouts(sur, train, DT, steps=200, iters_per_step=2, lr=5e-4, stat_steps=20)
    train.close()
    assert np.isfinite(losses).all()
    mean, std = sur.stats()
    trained = _heldout_loss(sur, _world(99))
    # the same network untrained, and with its output zeroed (the mean prediction)
    fresh = S.Surrogate(seed=5)
    fresh.set_stats(mean, std)
    untrained = _heldout_loss(fresh, _world(99))
    p = fresh.get_params()
    p["dec.2.W"][:] = 0.0
    p["dec.2.b"][:] = 0.0
    fresh.set_params(p)
    without = _heldout_loss(fresh, _world(99))
    assert trained < 0.2 * without, (trained, without)
    assert trained < untrained, (trained, untrained)


def test_fallback_reproduces_the_plain_run_and_no_fallback_keeps_learned_steps():
    sur = S.Surrogate(seed=6)
    plain = _world(7, 2)
    plain.run(DT, 20)
    learned = _world(7, 2)
    stats = S.run_learned(learned, sur, DT, 20, judge_every=5, bound=1e-300)
    assert stats["windows"] == 4 and stats["fallbacks"] == 4 and stats["plain_steps"] == 20
    for a, b, what in ((learned.positions(), plain.positions(), "x"),
                       (learned.velocities(), plain.velocities(), "v"),
                       (learned.densities(), plain.densities(), "rho")):
        assert_bits_equal(a, b, what)
    assert learned.t == plain.t
    keep = _world(7, 2)
    stats = S.run_learned(keep, sur, DT, 10, judge_every=5, bound=1e300)
    assert stats["fallbacks"] == 0 and stats["learned_steps"] == 10
    assert np.isfinite(keep.positions()).all()
    for w in (plain, learned, keep):
        w.close()
