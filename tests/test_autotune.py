"""The autotuner's coordinate descent and its tuning files, on a fake renderer (no GPU): the
fake's device time per sample is a known function of the launch settings, so the search must
end at its minimum, measure calls of several samples, and round-trip the stored JSON."""
import json

from xenon_b200 import autotune


class FakeRenderer:
    """Device ms per sample: a separable bowl over the tuning space, minimum at BEST."""
    BEST = {"refill": 16, "extend_blocks_per_sm": 8, "wave_paths": 1 << 22, "waves": 2, "graph": 1}

    def __init__(self):
        self.t = {k: v[0] for k, v in autotune.SPACE.items()}
        self.calls = []
        self._ms = 0.0

    def tuning(self):
        return dict(self.t)

    def set_tuning(self, **kw):
        self.t.update(kw)

    def render_range(self, cam, first, n):
        self.calls.append((first, n))
        cost = 3.0
        for k, want in self.BEST.items():
            vals = autotune.SPACE[k]
            cost += 0.1 * abs(vals.index(self.t[k]) - vals.index(want))
        self._ms = cost * n

    def stats(self):
        class S:
            pass
        s = S()
        s.last_ms = self._ms
        return s


def test_coordinate_descent_finds_the_minimum_and_measures_multi_sample_calls():
    r = FakeRenderer()
    res = autotune.autotune(r, None, "fake", calls=3, spp_per_call=4, save=False, log=lambda *_: None)
    for k, v in FakeRenderer.BEST.items():
        assert res["tuning"][k] == v, (k, res["tuning"][k])
    assert abs(res["ms_per_spp"] - 3.0) < 1e-9
    assert all(n == 4 for _, n in r.calls)
    # every measurement renders samples no other measurement used
    firsts = [f for f, _ in r.calls]
    assert len(firsts) == len(set(firsts))


def test_plain_workloads_leave_the_guided_knobs_alone():
    """guided_form changes nothing in a plain render, so a plain search must not move it (a
    noise 'gain' there would slow down guided renders that share the tuning)."""
    class Noisy(FakeRenderer):
        BEST = dict(FakeRenderer.BEST, guided_form=2)
    r = Noisy()
    res = autotune.autotune(r, None, "fake", calls=1, spp_per_call=1, save=False, log=lambda *_: None)
    assert res["tuning"]["guided_form"] == autotune.SPACE["guided_form"][0]
    r = Noisy()
    res = autotune.autotune(r, None, "fake", calls=1, spp_per_call=1, save=False, log=lambda *_: None, guided=True)
    assert res["tuning"]["guided_form"] == 2


def test_tuning_files_round_trip(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "TUNING_DIR", str(tmp_path))
    assert autotune.load_tuning("fake", gpu="G") is None
    p = autotune.tuning_path("fake", gpu="G")
    assert p.startswith(str(tmp_path))
    (tmp_path / "G").mkdir()
    with open(p, "w") as f:
        json.dump({"workload": "fake", "tuning": {"refill": 8}}, f)
    assert autotune.load_tuning("fake", gpu="G") == {"refill": 8}


def test_search_space_has_no_zero_values():
    # a zero field keeps the renderer's current value (xb_tuning), so it can never be a candidate
    for k, vals in autotune.SPACE.items():
        assert 0 not in vals, k
