"""Host logic of the autotuner (no GPU): the choice rule, the keys per particle order, and the
JSON cache (atomic write, per-GPU entries, application to a context)."""
import json

import openspacecharge_b200 as osc
from openspacecharge_b200 import autotune


class FakeCtx:
    def __init__(self):
        self.t = {}

    def set_tuning(self, k, v):
        self.t[k] = v


def test_choose_prefers_the_fastest_and_the_default_on_ties():
    assert autotune.choose({0: 1.0, 8: 0.5, 32: 0.7}) == 8
    assert autotune.choose({0: 1.0, 8: 1.0}) == 0


def test_keys_depend_on_particle_order_and_length():
    k_any = autotune.keys_for((128, 128, 256), osc.ORDER_ANY)
    assert "lines_nl_div:f32:L256" in k_any and "deposit_ctas_per_sm" in k_any and "deposit_run" not in k_any
    k_sorted = autotune.keys_for((64, 48, 96), osc.ORDER_CELL_SORTED, osc.PREC_FP64)
    assert "lines_nl_div:f64:L96" in k_sorted and "gather_run" in k_sorted
    assert k_any["zconv_engine:f32:L512"][1] == [0, 1, 2] and k_sorted["zconv_engine:f64:L192"][1] == [0, 2]
    assert all(cands for _, cands in k_sorted.values())


def test_cache_roundtrip_and_apply(tmp_path):
    p = str(tmp_path / "sub" / "autotune.json")
    assert autotune.load_cache(p) == {}
    autotune.save_cache({"GPU A": {"gather_run": {"value": 8, "ms": 0.1}, "lines_nl_div:f32:L256": {"value": 2}},
                         "GPU B": {"gather_run": {"value": 4}}}, p)
    assert json.load(open(p))["GPU A"]["gather_run"]["value"] == 8
    c = FakeCtx()
    applied = autotune.apply(c, path=p, gpu="GPU A")
    assert applied == {"gather_run": 8, "lines_nl_div:f32:L256": 2} and c.t == applied
    assert autotune.apply(FakeCtx(), path=p, gpu="GPU C") == {}


def test_cache_path_from_environment(monkeypatch, tmp_path):
    monkeypatch.setenv("OSC_TUNE_CACHE", str(tmp_path / "x.json"))
    assert autotune.cache_path() == str(tmp_path / "x.json")
    assert autotune.cache_path("/explicit.json") == "/explicit.json"
