"""Launch shapes change no result: the catalogue of the 64^3 snapshot with
thresholds that move most haloes to other tiers (wider CTAs, clusters from
2048 members) meets the parity bar against the default thresholds; the
tuner returns a valid setting whose catalogue it has checked."""
import pytest

from asohf_b200 import api, autotune as at, driver, synth

pytestmark = pytest.mark.gpu


def test_other_tiers_same_catalogue_and_tuner(gpu_lib):
    plan = driver.prepare(synth.generate("cfg1"))
    b = api.GpuBackend(0)
    ref = at.catalogue_of(plan, b, at.DEFAULTS)
    forced = {"tier1": 64, "tier2": 512, "cluster_min": 2048, "cluster_share": 1024}
    assert at.same_catalogue(ref, at.catalogue_of(plan, b, forced))
    space = {"tier1": [128, 256], "cluster_min": [16384, 32768]}
    best, ms, trials = at.tune_plan(plan, b, reps=1, space=space, rounds=1)
    assert at.valid(best) and ms > 0 and len(trials) >= 2
    assert at.same_catalogue(ref, at.catalogue_of(plan, b, best))
    at.apply(b.a, at.DEFAULTS)
