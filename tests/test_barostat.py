"""The Monte Carlo barostat (src/reference/barostat.ts:129-274, loop.ts:602-641)
and its screening network (no reference counterpart).

* One volume move on the GPU against the oracle: the same Threefry draws
  (threefry2x32([draw, seed], [0x6a09e667, 0]), loop.ts:614-622), the same
  molecule-centre scaling (barostat.ts:210), the oracle's f64 energies for
  the acceptance test.
* The network's CUDA gradient against the oracle's f64 reverse accumulation,
  and its training on the device.
* Delayed acceptance against the plain barostat on the same system: what
  the trained network saves (exact evaluations per attempt), and that the
  volume it samples agrees.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KB = 0.008314462618153242


def uniform(oracle, draw: int, seed: int) -> float:
    out = (C.c_uint32 * 2)()
    oracle.lib().orc_threefry2x32(draw, seed, 0x6A09E667, 0, 20, out)
    return (float(out[0] >> 9) + 0.5) * 2.0**-23


@pytest.mark.parametrize("seed", [3, 8, 21])
def test_one_volume_move_matches_oracle(oracle, seed):
    from mdb200 import steploop, synth

    system, state = synth.water_box(n_waters=700, width=2.8, seed=seed, grid=(28, 28, 28),
                                    barostat=(1.0, 300.0, 1))
    opts = steploop.RunOptions(seed=seed, mesh=(28, 28, 28))
    # the state right before the move: the same step without a barostat
    plain_sys, _ = synth.water_box(n_waters=700, width=2.8, seed=seed, grid=(28, 28, 28))
    before = steploop.StepLoop.from_parsed(plain_sys, state, opts)
    before.run(1)
    p1 = before.positions()
    before.destroy()
    loop = steploop.StepLoop.from_parsed(system, state, opts)
    loop.run(1)
    box_after, p_after = loop.box_vectors(), loop.positions()
    stats = loop.barostat_statistics()
    loop.destroy()
    assert stats["attempts"] == 1
    # the oracle's move
    box0 = np.asarray(state.box)
    volume = abs(np.linalg.det(box0))
    dv = 0.01 * volume * 2 * (uniform(oracle, 0, seed) - 0.5)
    scale = ((volume + dv) / volume) ** (1 / 3)
    trial = oracle.scale_molecules(system, p1, scale).reshape(-1, 3)
    e0, _ = oracle.potential(system, p1, box=box0, grid=(28, 28, 28), forces=False)
    e1, _ = oracle.potential(system, trial, box=box0 * scale, grid=(28, 28, 28), forces=False)
    kt = KB * 300.0
    n_mol = 700
    w = e1["potential"] - e0["potential"] + 1.0 * 0.06022140762081242 * dv - n_mol * kt * math.log((volume + dv) / volume)
    accept = not (w > 0 and uniform(oracle, 1, seed) > math.exp(-w / kt))
    print("seed", seed, "dV", dv, "w", w, "accepted", accept, "engine accepted", stats["accepted"])
    assert stats["accepted"] == int(accept)
    want_box = box0 * scale if accept else box0
    want_pos = trial if accept else p1
    assert np.allclose(box_after, want_box, rtol=0, atol=1e-12)
    assert np.abs(p_after - want_pos).max() < 1e-8


def test_network_gradient_matches_oracle(oracle):
    from mdb200 import steploop

    rng = np.random.default_rng(4)
    params = rng.normal(0, 0.3, steploop.MLP_PARAMS).astype(np.float32)
    # the kernels compute with BF16 weights: round to nearest even on the bits
    # so that both sides see the same values
    bits = params.view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    params = bits.astype(np.uint32).view(np.float32)
    x = rng.normal(size=(128, 16)).astype(np.float32)
    t = rng.normal(size=128).astype(np.float32)
    loss, g = steploop.mlp_gradient(params, x, t)
    want_loss, want = oracle.mlp_gradient(params, x, t)
    err = np.abs(g - want).max() / np.abs(want).max()
    print("loss", loss, want_loss, "grad max rel", err)
    assert abs(loss - want_loss) <= 1e-5 * want_loss
    assert err < 2e-5, err


def test_network_trains_on_the_device():
    from mdb200 import steploop

    rng = np.random.default_rng(9)
    x = rng.normal(size=(2048, 16)).astype(np.float32)
    t = (0.8 * x[:, 0] * x[:, 9] + np.sin(x[:, 1]) + 0.3 * x[:, 2] ** 2 - 0.5 * x[:, 3]).astype(np.float32)
    t = (t - t.mean()) / t.std()
    params, losses = steploop.mlp_fit(x, t, epochs=150, seed=1)
    print("loss first/last", losses[0], losses[-1])
    assert losses[-1] < 0.05 * losses[0] and losses[-1] < 0.05
    y = steploop.mlp_predict(params, x)
    assert np.mean((y - t) ** 2) < 0.06
    again, _ = steploop.mlp_fit(x, t, epochs=150, seed=1)
    assert np.array_equal(params, again)  # fixed-order reductions: training is reproducible


def test_delayed_acceptance_saves_exact_evaluations():
    """The same NPT water box with the plain barostat and with the screening
    network trained on its first 300 exact attempts: the network must reject
    some proposals on its own (fewer exact evaluations per attempt), stay
    within 1.5 kT RMS of the exact change (the limit above which the exact
    stage switches it off), and sample the same volume."""
    import time

    from mdb200 import steploop, synth

    system, state = synth.water_box(n_waters=884, width=3.0, seed=1, grid=(30, 30, 30), barostat=(1.0, 300.0, 4))
    results = {}
    for name, attempts in (("plain", 0), ("screened", 300)):
        loop = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(seed=2, surrogate_attempts=attempts))
        loop.run(1200)  # 300 attempts: the training set
        v = []
        t0 = time.perf_counter()
        start = loop.barostat_statistics()
        for _ in range(40):
            loop.run(40)
            v.append(abs(np.linalg.det(loop.box_vectors())))
        elapsed = time.perf_counter() - t0
        stats = loop.barostat_statistics()
        loop.destroy()
        n_att = stats["attempts"] - start["attempts"]
        exact = stats["exactEvaluations"] - start["exactEvaluations"]
        results[name] = dict(volume=float(np.mean(v)), exact_per_attempt=exact / n_att, seconds=elapsed, **stats)
        print(name, results[name])
    s, p = results["screened"], results["plain"]
    assert p["exact_per_attempt"] == 2.0
    assert s["surrogateActive"] and s["trainingSamples"] == 300
    assert s["screened"] > 0
    assert s["exact_per_attempt"] < 0.9 * p["exact_per_attempt"]
    assert s["surrogateRms"] < 1.5 * KB * 300.0
    assert abs(s["volume"] - p["volume"]) < 0.03 * p["volume"]


def test_screened_and_plain_barostat_sample_the_same_volume_distribution():
    """Detailed balance is unchanged by the screening stage: from the same
    equilibrated state, the plain and the screened barostat give the same
    mean volume within four combined standard errors (block averages of 20
    blocks over 20,000 attempts each), and volume fluctuations within 25%."""
    from mdb200 import steploop, synth
    from mdb200.system import State

    system, state = synth.water_box(n_waters=884, width=3.0, seed=1, grid=(30, 30, 30), barostat=(1.0, 300.0, 4))
    warm = steploop.StepLoop.from_parsed(system, state, steploop.RunOptions(seed=5))
    warm.run(20000)
    start = State(positions=warm.positions(), box=warm.box_vectors(), velocities=warm.velocities(), step=warm.steps)
    warm.destroy()
    samples = {}
    for name, attempts, seed in (("plain", 0, 11), ("screened", 300, 12)):
        loop = steploop.StepLoop.from_parsed(system, start,
                                             steploop.RunOptions(seed=seed, surrogate_attempts=attempts))
        loop.run(1200)  # the screened arm's 300 training attempts; the same steps for the plain one
        v = []
        for _ in range(2000):
            loop.run(40)
            v.append(abs(np.linalg.det(loop.box_vectors())))
        stats = loop.barostat_statistics()
        loop.destroy()
        samples[name] = np.array(v)
        print(name, float(np.mean(v)), float(np.std(v)), stats)
    means, errors = {}, {}
    for name, v in samples.items():
        blocks = v.reshape(20, -1).mean(axis=1)
        means[name] = float(v.mean())
        errors[name] = float(blocks.std(ddof=1) / math.sqrt(len(blocks)))
    gap = abs(means["screened"] - means["plain"])
    bound = 4.0 * math.hypot(errors["screened"], errors["plain"])
    print("mean volumes", means, "standard errors", errors, "gap", gap, "bound", bound)
    assert gap < bound
    ratio = samples["screened"].std() / samples["plain"].std()
    assert 0.75 < ratio < 1.25, ratio


def test_batched_barostat_rounds_move_each_system_as_it_moves_alone():
    """Systems whose barostats are due together attempt in one round -- one
    evaluation of the engine for their current energies, one for their
    proposals -- and each draws from its own counter, so a system in a batch
    makes exactly the moves it makes alone: positions, boxes and barostat
    counts bit-identical."""
    from mdb200 import steploop, synth

    members = [synth.water_box(n_waters=700, width=2.8, seed=4, grid=(28, 28, 28), barostat=(1.0, 300.0, 5)),
               synth.water_box(n_waters=900, width=3.1, seed=5, grid=(32, 32, 32), barostat=(1.0, 300.0, 5))]
    opts = steploop.RunOptions(seed=9)
    alone = []
    for system, state in members:
        loop = steploop.StepLoop.from_parsed(system, state, opts)
        loop.run(200)
        alone.append((loop.positions(), loop.box_vectors(), loop.barostat_statistics(), loop.verlet_flags()))
        loop.destroy()
    batch = steploop.StepLoop.batch([m[0] for m in members], [m[1] for m in members], opts)
    batch.run(200)
    for k, (p, b, st, fl) in enumerate(alone):
        got = batch.barostat_statistics(k)
        print("system", k, "alone", st, fl, "batch", got)
        assert got["attempts"] == st["attempts"] == 40 and got["accepted"] == st["accepted"]
        assert np.array_equal(batch.box_vectors(k), b)
        assert np.array_equal(batch.positions(k), p)
        assert st["accepted"] >= 5
    batch.destroy()
