"""Launch-shape tuner for the per-halo kernels.

The halo and subhalo kernels (the replacements of HALOFIND_PARTICLES,
haloes_particles.f:578-1411, and SUBSTRUCTURE_PARTICLES, substructure.f:756)
run in size tiers: one CTA of 32, 128 or 256 threads per halo, or a
thread-block cluster for the largest.  The member counts that separate the
tiers are setters of the library (``Asohf.set_group_tiers``,
``set_cluster_threshold``, ``set_cluster_share``).  Which thresholds are
fastest depends on the snapshot's halo-size distribution and on how the
concurrent tiers share the SMs, so ``tune`` times the caller's own plan on
the device for a small grid of settings, one setter at a time with the
others held (coordinate descent), and returns the fastest.  ``apply`` sets a
choice on a backend; ``save`` and ``load`` keep it per workload signature in
a JSON file.

A setting changes launch shapes only: in every tier the kernels give the
same integer fields and ID lists, and float fields within float32 rounding
of the reduction order (1e-5 relative, the parity bar against the oracle).
``tune_plan`` checks the chosen setting against the default setting's
catalogue by that bar (``check=True``) and keeps the defaults when it fails.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

DEFAULTS = {"tier1": 256, "tier2": 2048, "cluster_min": 32768, "cluster_share": 32768}
SPACE = {
    "tier1": [128, 256, 512],
    "tier2": [1024, 2048, 4096],
    "cluster_min": [16384, 32768, 65536, 131072],
    "cluster_share": [16384, 32768, 65536],
}
_INT_FIELDS = ("realclus", "dmpclus")
_FLOAT_FIELDS = ("masa", "radio", "clusrx", "clusry", "clusrz", "msub", "rsub")


def valid(p: dict) -> bool:
    """tier1 <= tier2 <= cluster_min (the setters refuse tier2 < tier1)."""
    return 0 < p["tier1"] <= p["tier2"] <= p["cluster_min"] and p["cluster_share"] > 0


def apply(lib, p: dict) -> None:
    """Sets the four thresholds on an ``api.Asohf`` handle."""
    lib.set_group_tiers(int(p["tier1"]), int(p["tier2"]))
    lib.set_cluster_threshold(int(p["cluster_min"]))
    lib.set_cluster_share(int(p["cluster_share"]))


def signature(plan) -> str:
    """The workload a choice belongs to: configuration, particles, grid,
    levels and candidate haloes."""
    cfg = plan.snap.cfg
    return f"{cfg.name}:n{plan.snap.x.shape[0]}:nx{cfg.nx}:nl{cfg.nl}:c{len(plan.cand.clusrx)}"


def device_timer(plan, backend, with_subs: bool = True, reps: int = 3):
    """A timer for ``tune``: median device time (ms) of ``reps`` runs of the
    hot path after one untimed run.  The backend is set to run on torch's
    current stream, where the timing events are recorded."""
    import torch
    from . import driver

    st = torch.cuda.current_stream()
    backend.a.set_stream(st.cuda_stream)

    def run():
        return driver.execute(plan, backend, with_subs=with_subs, download=False)

    def timer(p: dict) -> float:
        apply(backend.a, p)
        run()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            run()
            e1.record(st)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    return timer


def catalogue_of(plan, backend, p: dict, with_subs: bool = True) -> dict:
    """The catalogue columns a setting produces (host copies)."""
    from . import driver

    apply(backend.a, p)
    r = driver.execute(plan, backend, with_subs=with_subs, download=True)
    n = int(r.cat.nclus)
    out = {f: _host(getattr(r.cat, f)[:n]) for f in _INT_FIELDS + _FLOAT_FIELDS}
    out["pph"] = _host(r.pph)
    return out


def _host(a) -> np.ndarray:
    """A host copy of a numpy array or a torch tensor (device tensors of the
    device-resident backend included)."""
    if hasattr(a, "detach") and hasattr(a, "cpu"):
        return a.detach().cpu().numpy().copy()
    return np.array(a)


def same_catalogue(a: dict, b: dict, rtol: float = 1e-5) -> bool:
    """Integer fields and the ID stream equal, floats within rtol."""
    if any(not np.array_equal(a[k], b[k]) for k in _INT_FIELDS + ("pph",)):
        return False
    for k in _FLOAT_FIELDS:
        x, y = a[k].astype(np.float64), b[k].astype(np.float64)
        if x.shape != y.shape or not np.all(np.abs(x - y) <= rtol * np.maximum(np.abs(x), np.abs(y)) + 1e-30):
            return False
    return True


def tune(timer, space: dict | None = None, start: dict | None = None, rounds: int = 2, verify=None):
    """Coordinate descent over ``space`` from ``start`` (the defaults).

    timer(p) -> ms for a setting p; verify(p) -> bool, called once on the
    chosen setting when it differs from the start (the catalogue check): a
    setting that fails it is refused and the start is returned.
    Returns (setting, its time, every trial as (setting, ms)).
    """
    space = space or SPACE
    best = dict(start or DEFAULTS)
    trials = []
    seen = {}

    def measure(p):
        key = tuple(sorted(p.items()))
        if key not in seen:
            seen[key] = timer(p)
            trials.append((dict(p), seen[key]))
        return seen[key]

    best_ms = measure(best)
    for _ in range(rounds):
        changed = False
        for name, values in space.items():
            for v in values:
                if v == best[name]:
                    continue
                p = dict(best, **{name: v})
                if not valid(p):
                    continue
                ms = measure(p)
                if ms < best_ms:
                    best, best_ms, changed = p, ms, True
        if not changed:
            break
    start = dict(start or DEFAULTS)
    if verify is not None and best != start and not verify(best):
        return start, measure(start), trials
    return best, best_ms, trials


def tune_plan(plan, backend, with_subs: bool = True, reps: int = 3, space: dict | None = None,
              rounds: int = 2, check: bool = True):
    """``tune`` on the device with the caller's plan; the backend keeps the
    chosen setting.  Returns (setting, ms, trials)."""
    timer = device_timer(plan, backend, with_subs, reps)
    verify = None
    if check:
        ref = catalogue_of(plan, backend, DEFAULTS, with_subs)

        def verify(p):
            return same_catalogue(ref, catalogue_of(plan, backend, p, with_subs))
    best, ms, trials = tune(timer, space, DEFAULTS, rounds, verify)
    apply(backend.a, best)
    return best, ms, trials


def save(path: str, sig: str, p: dict, ms: float) -> None:
    """Keeps a choice for a workload signature (other entries kept)."""
    data = {}
    if os.path.exists(path):
        with open(path) as f:
            data = json.load(f)
    data[sig] = {"setting": p, "ms": ms, "time": time.strftime("%Y-%m-%dT%H:%M:%S")}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def load(path: str, sig: str):
    """The kept choice for a signature, or None."""
    if not os.path.exists(path):
        return None
    with open(path) as f:
        e = json.load(f).get(sig)
    if not e:
        return None
    p = e["setting"]
    return p if valid(p) else None
