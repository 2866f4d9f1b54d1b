"""The launch-shape tuner's search, setting validity, setters and cache
(host logic, a synthetic cost in place of device timings)."""
from asohf_b200 import autotune as at


def cost(p):
    """A separable bowl with its minimum at tier1 512, tier2 1024,
    cluster_min 65536, cluster_share 16384."""
    return (abs(p["tier1"] - 512) / 128 + abs(p["tier2"] - 1024) / 1024 + abs(p["cluster_min"] - 65536) / 16384
            + abs(p["cluster_share"] - 16384) / 16384 + 100.0)


def test_descent_finds_the_minimum_and_measures_each_setting_once():
    calls = []

    def timer(p):
        calls.append(tuple(sorted(p.items())))
        return cost(p)
    best, ms, trials = at.tune(timer)
    assert best == {"tier1": 512, "tier2": 1024, "cluster_min": 65536, "cluster_share": 16384}
    assert ms == cost(best)
    assert len(calls) == len(set(calls)) == len(trials)
    assert all(at.valid(p) for p, _ in trials)


def test_defaults_kept_when_nothing_is_faster_and_no_check_needed():
    verified = []
    best, _, trials = at.tune(lambda p: 1.0 + 0.0 * p["tier1"] if p == at.DEFAULTS else 2.0,
                              verify=lambda p: verified.append(p) or True)
    assert best == at.DEFAULTS and not verified and len(trials) > 1


def test_a_setting_that_changes_the_catalogue_is_refused():
    best, ms, _ = at.tune(cost, verify=lambda p: False)
    assert best == at.DEFAULTS and ms == cost(at.DEFAULTS)


def test_catalogue_bar():
    import numpy as np
    a = {k: np.arange(5, dtype=np.int32) for k in at._INT_FIELDS + ("pph",)}
    a.update({k: np.linspace(1, 2, 5).astype(np.float32) for k in at._FLOAT_FIELDS})
    b = {k: v.copy() for k, v in a.items()}
    assert at.same_catalogue(a, b)
    b["masa"][2] *= np.float32(1 + 2e-6)      # float rounding: accepted
    assert at.same_catalogue(a, b)
    b["masa"][2] *= np.float32(1 + 1e-4)
    assert not at.same_catalogue(a, b)
    b = {k: v.copy() for k, v in a.items()}
    b["pph"][0] = 9                            # a different member: refused
    assert not at.same_catalogue(a, b)


def test_valid_and_apply():
    assert at.valid(at.DEFAULTS)
    assert not at.valid(dict(at.DEFAULTS, tier1=4096))        # tier1 > tier2
    assert not at.valid(dict(at.DEFAULTS, tier2=65536))       # tier2 > cluster_min

    class Lib:
        def __init__(self):
            self.calls = []

        def set_group_tiers(self, a, b):
            self.calls.append(("tiers", a, b))

        def set_cluster_threshold(self, a):
            self.calls.append(("thr", a))

        def set_cluster_share(self, a):
            self.calls.append(("share", a))
    lib = Lib()
    at.apply(lib, dict(at.DEFAULTS, tier1=128))
    assert lib.calls == [("tiers", 128, 2048), ("thr", 32768), ("share", 32768)]


def test_cache_round_trip(tmp_path):
    path = str(tmp_path / "tune.json")
    assert at.load(path, "a") is None
    at.save(path, "a", at.DEFAULTS, 12.5)
    p = dict(at.DEFAULTS, cluster_min=65536)
    at.save(path, "b", p, 10.0)
    assert at.load(path, "a") == at.DEFAULTS and at.load(path, "b") == p and at.load(path, "c") is None


def test_host_copies_of_tensors():
    import numpy as np
    import torch
    t = torch.arange(4, dtype=torch.int32)
    h = at._host(t)
    assert isinstance(h, np.ndarray) and h.tolist() == [0, 1, 2, 3]
    a = np.arange(3)
    assert at._host(a) is not a and at._host(a).tolist() == [0, 1, 2]



def test_signature_names_the_workload():
    from types import SimpleNamespace
    import numpy as np
    cfg = SimpleNamespace(name="cfgX", nx=64, nl=3)
    plan = SimpleNamespace(snap=SimpleNamespace(cfg=cfg, x=np.zeros(10)), cand=SimpleNamespace(clusrx=np.zeros(7)))
    assert at.signature(plan) == "cfgX:n10:nx64:nl3:c7"
