"""CPU tests of the launch planner's selection logic (stratiflow_b200.autotune):
the search, the noise margin, the candidate space and the plan cache, with a
fake timing function in place of the device."""
import json

from stratiflow_b200 import autotune as A


def _cost(best, base=1.0, step=0.1):
    """A separable cost with its minimum at `best`."""
    def measure(s):
        c = base
        for k, v in best.items():
            c += step * abs(A.space(128, 384)[k].index(s[k]) - A.space(128, 384)[k].index(v))
        return c
    return measure


def test_search_finds_the_fastest_settings():
    best = {"xkernel": 0, "xy_bands": 6, "xslabs": 2, "z_chunks": 16, "xgroups": 16, "zkernel": 1}
    got, log = A.search(_cost(best), A.space(128, 384))
    assert got == best
    assert log[0][0] == {"xkernel": 1, "xy_bands": 1, "xslabs": 0, "z_chunks": 0, "xgroups": 0, "zkernel": 2}   # starts from the defaults


def test_search_keeps_the_default_within_the_noise_margin():
    def measure(s):   # every other value is 1% faster: not enough to switch
        return 0.99 if s != {"xkernel": 1, "xy_bands": 1, "xslabs": 0, "z_chunks": 0, "xgroups": 0, "zkernel": 2} else 1.0
    got, _ = A.search(measure, A.space(128, 384))
    assert got == {"xkernel": 1, "xy_bands": 1, "xslabs": 0, "z_chunks": 0, "xgroups": 0, "zkernel": 2}


def test_each_setting_is_measured_once():
    calls = []
    best = {"xkernel": 1, "xy_bands": 2, "xslabs": 6, "z_chunks": 8, "xgroups": 8, "zkernel": 0}
    f = _cost(best)
    A.search(lambda s: (calls.append(tuple(sorted(s.items()))), f(s))[1], A.space(128, 384))
    assert len(calls) == len(set(calls))


def test_space_depends_on_the_grid():
    two = A.space(1, 128)
    assert two["xy_bands"] == [A.DEFAULTS["xy_bands"]]     # no y transforms in 2D
    assert A.space(1, 16)["z_chunks"] == [0, 8]              # 16 chunks need 32 levels
    assert 16 in A.space(128, 384)["z_chunks"]
    assert two["xkernel"] == [1] and A.space(128, 384)["xkernel"] == [1, 0]   # 3D only


def test_plan_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "plans.json"
    monkeypatch.setenv("SF_PLAN_CACHE", str(path))
    A._memory.clear()
    key = A.plan_key("B200", 256, 128, 384, 1, "step")
    assert A.lookup(key) is None
    A.store(key, {"xkernel": 0, "xy_bands": 3, "xslabs": 6, "z_chunks": 8, "xgroups": 16, "zkernel": 1})
    assert json.load(open(path))[key]["xy_bands"] == 3
    A._memory.clear()
    assert A.lookup(key) == {"xkernel": 0, "xy_bands": 3, "xslabs": 6, "z_chunks": 8, "xgroups": 16, "zkernel": 1}


class _FakeSolver:
    N1, N2, N3, nrun, device = 64, 32, 64, 1, 0

    def __init__(self):
        self.applied = {}
        self.state = object()

    def set_xpass_kernel(self, v): self.applied["xkernel"] = v
    def set_xpass_slabs(self, v): self.applied["xslabs"] = v
    def set_xy_bands(self, v): self.applied["xy_bands"] = v
    def set_z_chunks(self, v): self.applied["z_chunks"] = v
    def set_xpass_groups(self, v): self.applied["xgroups"] = v
    def set_z_kernel(self, v): self.applied["zkernel"] = v
    def get_state_kept(self): return self.state
    def set_state_kept(self, st): assert st is self.state
    def TimeStep(self, n=1): pass
    def synchronize(self): pass


def test_tune_applies_and_caches_the_plan(tmp_path, monkeypatch):
    monkeypatch.setenv("SF_PLAN_CACHE", str(tmp_path / "plans.json"))
    A._memory.clear()
    s = _FakeSolver()
    best, log = A.tune(s, steps=1)
    assert log and s.applied == best
    s2 = _FakeSolver()
    again, log2 = A.tune(s2, steps=1)
    assert again == best and log2 == [] and s2.applied == best   # from the cache

