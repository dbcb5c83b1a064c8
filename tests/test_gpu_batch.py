"""Batched stepping (many lattices in one replayed step graph, every launch mode) gives
the same populations, fields and breakthrough series as stepping each
lattice on its own (run with -m gpu)."""
import numpy as np
import pytest

from fluidmaxxer_b200 import lattice, problems

pytestmark = pytest.mark.gpu


def small_samples(count=5, seed=77):
    """Uneven Bernoulli samples with drawn Langmuir parameters (the batch
    workload's generator at small edges)."""
    return problems.batch_samples(seed=seed, count=count, edges=(16, 24, 32, 40), steps=60)


@pytest.mark.parametrize("precision,mode", [("f32", 0), ("f32", 1), ("f32", 2), ("f32", 3), ("f64", 1), ("f16", 2),
                                            ("f16q", 1), ("f16", 3), ("f32", None)])
def test_batch_equals_individual_steps(precision, mode):
    ps = small_samples()
    solo = [lattice.from_problem(p, precision) for p in ps]
    for L in solo:
        L.step(61)
    bat = [lattice.from_problem(p, precision) for p in ps]
    B = lattice.Batch(bat)
    if mode is not None:   # None: the default mode of a new batch
        B.set_config(block=128, cells_per_thread=2, prefetch=1, mode=mode)
    B.step(3)        # single launches up to the graph boundary
    B.step(40)       # graph replays + remainder
    B.step(18)
    B.synchronize()
    for a, b in zip(solo, bat):
        sa, sb = a.get_state(), b.get_state()
        for k in ("f", "g", "phi", "q"):
            assert np.array_equal(sa[k], sb[k]), k
        assert np.allclose(a.breakthrough(), b.breakthrough(), rtol=1e-12, atol=0.0)   # FP64 sum order
        assert a.step_count == b.step_count == 61
    B.close()


@pytest.mark.parametrize("mode", [0, 3])
def test_batch_porous_equals_individual_steps(mode):
    # porous-BGK lattices of different sizes and porosity fields; six of
    # them, so mode 3 puts more than one lattice on a forked stream
    ps = [problems.smooth_porous(seed=900 + i, nx=16 + 8 * (i % 3), ny=16, nz=12 + 4 * (i % 2), steps=45)
          for i in range(6)]
    solo = [lattice.from_problem(p, "f32") for p in ps]
    for L in solo:
        L.step(45)
    bat = [lattice.from_problem(p, "f32") for p in ps]
    B = lattice.Batch(bat)
    B.set_config(block=256, cells_per_thread=1, prefetch=0, mode=mode)
    B.step(45)
    B.synchronize()
    for a, b in zip(solo, bat):
        sa, sb = a.get_state(), b.get_state()
        for k in ("f", "g", "phi", "q"):
            assert np.array_equal(sa[k], sb[k]), k
        assert np.allclose(a.breakthrough(), b.breakthrough(), rtol=1e-12, atol=0.0)
    B.close()


def test_batch_autotune_restores_state():
    ps = small_samples(count=3, seed=78)
    ref = [lattice.from_problem(p, "f32") for p in ps]
    for L in ref:
        L.step(20)
    bat = [lattice.from_problem(p, "f32") for p in ps]
    B = lattice.Batch(bat)
    B.step(10)
    cfg = B.autotune(trial_steps=2)
    assert cfg["block"] in (128, 256) and 1 <= cfg["cells_per_thread"] <= 4 and cfg["mode"] in (0, 1, 2, 3)
    B.step(10)
    B.synchronize()
    for a, b in zip(ref, bat):
        assert np.array_equal(a.get_state()["f"], b.get_state()["f"])
    B.close()


def test_batch_rejects_mixed_setups():
    ps = small_samples(count=2, seed=79)
    a = lattice.from_problem(ps[0], "f32")
    b = lattice.from_problem(ps[1], "f64")
    with pytest.raises(lattice._abi.FmError):
        lattice.Batch([a, b])
