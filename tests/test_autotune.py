"""The in-project autotuner (ablsteadyrans_b200.autotune): candidate
enumeration, the choice of the fastest, the per-shape cache (CPU), and on
the GPU one tuning of a tile that leaves the solve's state untouched."""
import json

import numpy as np
import pytest

from ablsteadyrans_b200 import autotune


def test_candidates_start_with_the_defaults_and_drop_no_op_combinations():
    cands = autotune.candidates()
    assert cands[0] == {"LINE_VARIANT": 0, "LINE_SEGMENT": 0, "MG_FUSED_RELAX": 0}
    keys = [json.dumps(c, sort_keys=True) for c in cands]
    assert len(keys) == len(set(keys))
    # the segment length does nothing with the sequential sweep and the two-launch relaxation
    assert {"LINE_VARIANT": 4, "LINE_SEGMENT": 4, "MG_FUSED_RELAX": 0} not in cands
    assert {"LINE_VARIANT": 4, "LINE_SEGMENT": 0, "MG_FUSED_RELAX": 0} in cands
    assert len(cands) == 2 * 3 * 2 - 2


def test_best_takes_the_fastest_and_keeps_the_earlier_on_ties():
    a, b, c = {"x": 1}, {"x": 2}, {"x": 3}
    assert autotune.best([(a, 2.0), (b, 1.0), (c, 1.5)]) == b
    assert autotune.best([(a, 1.0), (b, 1.0)]) == a
    with pytest.raises(ValueError):
        autotune.best([])


def test_shape_key_and_the_cache_file(tmp_path):
    from ablsteadyrans_b200 import workloads
    inst = workloads.tile(64, 48, 3)
    key = autotune.shape_key(inst.grid, inst.options, inst.physics)
    assert key.startswith("64x64x48:px0py0:prec1:")
    path = str(tmp_path / "tune.json")
    t = autotune.Autotuner(path)
    t.cache[key] = {"choice": {"LINE_VARIANT": 4}, "ms": {}}
    t.save()
    t2 = autotune.Autotuner(path)
    assert t2.cache[key]["choice"] == {"LINE_VARIANT": 4}


@pytest.mark.gpu
def test_gpu_autotuner_picks_a_candidate_and_restores_the_state(ctx, tmp_path):
    """Tuning a tile times every candidate on a copy of the state: the
    state is bit-identical afterwards, the choice is one of the candidates
    and is applied to the context, and the second call for the same shape
    comes from the cache."""
    import ablsteadyrans_b200 as gb
    import oracle
    from ablsteadyrans_b200 import workloads
    from ablsteadyrans_b200.simplec import DeviceCase, SimplecStage
    inst = workloads.tile(64, 48, 3)
    J, ax, ay, az, _ = oracle.metrics(inst.grid, inst.z)
    dc = DeviceCase(inst.grid, inst.z, J, ax, ay, az, inst.nu, inst.gamma_theta, inst.gamma_tke, inst.q, inst.z0map)
    st = SimplecStage(ctx, dc, inst.bc, inst.physics, inst.options)
    try:
        st.fill_ghosts()
        before = {f: dc.host(f) for f in dc.q}
        tuner = autotune.Autotuner(str(tmp_path / "tune.json"), iterations=2)
        choice, timings = tuner.tune(st)
        assert choice in autotune.candidates()
        assert len(timings) == len(autotune.candidates()) and all(ms > 0 for _, ms in timings)
        for f in dc.q:
            assert np.array_equal(dc.host(f), before[f]), f
        again, none = tuner.tune(st)
        assert again == choice and none is None
    finally:
        for name in autotune.CANDIDATES:
            ctx.tune(getattr(gb, "TUNE_" + name), 0)
        st.close()


def test_sweep_key_orders_systems_and_separates_precision_and_sweeps():
    """The batched sweep's cache key lists the systems' extents in a fixed
    order (the same batch in another order hits the same entry) and keeps
    FP64 and FP32, and different sweep counts, apart."""
    import torch
    from helpers import Grid
    from ablsteadyrans_b200.autotune import sweep_key
    a, b = Grid(8, 6, 5, 1.0, 1.0, 1.0), Grid(4, 4, 9, 1.0, 1.0, 1.0)
    d64, d32 = torch.zeros(1, dtype=torch.float64), torch.zeros(1, dtype=torch.float32)
    s1 = [(a, 1, d64), (b, 4, d64)]
    s2 = [(b, 4, d64), (a, 1, d64)]
    assert sweep_key(s1, 4) == sweep_key(s2, 4)
    assert sweep_key(s1, 4) != sweep_key(s1, 3)
    assert sweep_key(s1, 4) != sweep_key([(a, 1, d32), (b, 4, d32)], 4)
    assert "9x6x5" in sweep_key(s1, 4) and "4x4x10" in sweep_key(s1, 4)
