"""Continuous batching: every result is the same alone and in the mix; the HBM
budget bounds concurrency; the autotuner records a valid tile width."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup():
    import torch
    from aapm_lowdosectimagerecon_competition_b200 import serve
    assert torch.cuda.is_available()
    dev = torch.device("cuda", 0)
    sizes = [(64, 4, 60), (96, 12, 90), (80, 8, 72), (64, 9, 120), (72, 5, 66)]
    insts = [serve.make_instance(N, Z, P, seed=20 + i, device=dev, iters=3, numOfOS=4)
             for i, (N, Z, P) in enumerate(sizes)]
    return torch, serve, dev, insts


def _images(engine):
    return {f["tag"]: f["image"].numpy().copy() for f in engine.finished}


def test_each_result_is_the_same_alone_and_in_the_mix(setup):
    torch, serve, dev, insts = setup
    alone = {}
    for inst in insts:
        e = serve.Engine(device=0, max_active=1)
        e.submit(inst)
        e.drain()
        alone.update(_images(e))
    mix = serve.Engine(device=0, max_active=4)
    out = serve.run_batch(insts, mix)
    assert out["instances"] == len(insts) and mix.peak_active > 1
    got = _images(mix)
    for tag, img in alone.items():
        np.testing.assert_array_equal(got[tag], img)


def test_engine_equals_one_call_api(setup):
    torch, serve, dev, insts = setup
    from aapm_lowdosectimagerecon_competition_b200 import dd2
    inst = insts[1]
    s = inst.scan
    e = serve.Engine(device=0, max_active=2)
    e.submit(inst)
    e.drain()
    ref = dd2.OSSART_AAPM(inst.proj_host.numpy(), s.hangs(), np.zeros((s.YN, s.XN, s.SLN), np.float32),
                          s.conf(), inst.iters, s.numOfOS, inst.mask, s.useFISTA, s.nonneg, sat="hilo",
                          back="adj")
    np.testing.assert_array_equal(e.finished[0]["image"].numpy(), ref)


def test_budget_bounds_concurrency(setup):
    torch, serve, dev, insts = setup
    probe = serve.Engine(device=0)
    need = sorted(probe.estimate(i) for i in insts)
    budget = need[-1] + 0.5 * need[0]  # the largest fits, never two of the larger ones
    e = serve.Engine(device=0, budget_bytes=budget, max_active=4)
    out = serve.run_batch(insts, e)
    assert out["instances"] == len(insts)
    assert e.peak_used <= budget and 1 <= e.peak_active < len(insts)
    with pytest.raises(ValueError):
        serve.Engine(device=0, budget_bytes=0.5 * need[-1]).submit(max(insts, key=probe.estimate))


def test_tuner_records_a_valid_width(setup):
    torch, serve, dev, insts = setup
    from aapm_lowdosectimagerecon_competition_b200._lib import load
    lib = load()
    t = serve.TileTuner()
    zl, nz = t.tune(N=64, Z=32, P=48, device=dev, reps=1)
    assert zl in (1, 2, 4, 8) and nz == 0 and lib.ddfan_tune_get_zl(8) == zl
    lib.ddfan_tune_set_zl(8, 0)


def test_tuner_records_a_shape_in_the_direct_mode(setup, tmp_path):
    torch, serve, dev, insts = setup
    from aapm_lowdosectimagerecon_competition_b200._lib import load
    lib = load()
    cache = str(tmp_path / "tiles.json")
    t = serve.TileTuner(cache_path=cache, sat="direct", back="ref")
    zl, nz = t.tune(N=64, Z=64, P=48, device=dev, reps=1)
    # 16 blocks: widths 8, 4, 2, 1 with every z-tiles-per-thread count that fits
    assert len(t.timings[16]) == 2 + 3 + 3 + 3
    assert zl in (1, 2, 4, 8) and nz in (1, 2, 4)
    assert lib.ddfan_tune_get_zl(16) == zl and lib.ddfan_tune_get_nz(16) == nz
    t.save()
    lib.ddfan_tune_set_zl(16, 0)
    lib.ddfan_tune_set_nz(16, 0)
    assert lib.ddfan_tune_get_nz(16) == 4
    serve.TileTuner(cache_path=cache, sat="direct")  # re-applies the cached record
    assert lib.ddfan_tune_get_zl(16) == zl and lib.ddfan_tune_get_nz(16) == nz
    lib.ddfan_tune_set_zl(16, 0)
    lib.ddfan_tune_set_nz(16, 0)
