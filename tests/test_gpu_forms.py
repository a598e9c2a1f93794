"""The precision form on a small channel: FP64 state / RK / pressure with
FP32 fluxes is closer to the all-FP64 run than the all-FP32 pipeline, with
drift figures and throughput reported for every pipeline."""

import numpy as np
import pytest

from opendynamo_b200.forms.precision import precision_study


@pytest.mark.gpu
def test_precision_study_small():
    out = precision_study(n=6, steps=40, dt=1e-3, chunk=20)
    p = out["pipelines"]
    assert p["f64"]["rel_l2_vs_f64"] == [0.0] * 5
    mixed, f32 = np.array(p["mixed"]["rel_l2_vs_f64"]), np.array(p["f32"]["rel_l2_vs_f64"])
    assert np.all(mixed < 1e-5) and np.all(f32 < 1e-3)
    assert np.all(mixed <= f32), (mixed, f32)
    for name in ("f64", "mixed", "f32"):
        assert np.isfinite(p[name]["ke_drift"]) and np.isfinite(p[name]["enstrophy_drift"])
        assert p[name]["gdof_stage_s"] > 0
    assert p["mixed"]["ke_max_rel_dev_vs_f64"] <= p["f32"]["ke_max_rel_dev_vs_f64"] * 1.01 + 1e-12
