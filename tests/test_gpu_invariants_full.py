"""The hot path at the benchmark size: the 512^3-particle snapshot (250
Mpc/h, 6 AMR levels, 2e5 haloes and their subhaloes) run through the
device-resident path.

Size-independent checks: mass conservation of the base-grid deposit, the
x-slab sort (sorted store, consistent NDMPART_X), and the catalogue
(consistent INDCS ranges over the ID stream, IDs valid and unique within
each halo, bound counts above MIN_NUM_PART, positive masses and radii,
centres in the box).

Parity on a window: the oracle would take too long on every halo, so it
reruns, on the same x-sorted store, a seeded window of rows from every
HALOFIND_PARTICLES and SUBSTRUCTURE_PARTICLES call of the run -- the 20
largest of each call, every halo of the thread-block-cluster tier (32768
members and more) and 200 others drawn at random -- and each row must equal
the device's (integer fields and ID lists identical, floats within 1e-5),
unless the oracle counted a particle test within a relative 1e-6 of its
threshold in that row.  The margin counts are printed with the result."""
import numpy as np
import pytest

from asohf_b200 import api, driver, grid, synth
from tests import window_parity as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def run512(gpu_lib):
    import torch
    cfg = synth.CONFIGS["cfg4"]
    snap = synth.generate_fast(cfg, device="cuda:0", keep_on_device=True)
    plan = driver.prepare(snap)
    b = api.DeviceBackend(0)
    b.a.set_stream(torch.cuda.current_stream().cuda_stream)
    rec = W.Recorder(b)
    r = driver.execute(plan, rec, with_subs=True, download=False)
    torch.cuda.synchronize()
    b.calls = rec.calls
    return cfg, snap, plan, b, r


def test_density_conserves_mass(run512):
    import torch
    cfg, snap, plan, b, r = run512
    cos = plan.cos
    u1, _ = b.density(cfg.nx, np.float32(cfg.lado0), plan.dx, cos["rote"], cos["rete"], r.npart_esp,
                      plan.mesh)
    torch.cuda.synchronize()
    dx = np.float32(plan.dx)
    denbas = float(dx * dx * dx * np.float32(cos["rote"]) * np.float32(cos["rete"]) ** 3)
    total = float(u1.double().sum()) * denbas
    mass = float(snap.m.double().sum())
    # the 27 kernel weights sum to 1 up to float32 rounding
    assert abs(total - mass) <= 1e-5 * mass


def test_x_sort_and_slab_table(run512):
    import torch
    cfg, snap, plan, b, r = run512
    n = snap.x.shape[0]
    out = [torch.empty(n, dtype=torch.float32, device="cuda:0") for _ in range(7)] + \
          [torch.empty(n, dtype=torch.int32, device="cuda:0")]
    b.a.download_particles(out)
    torch.cuda.synchronize()
    x = out[0]
    assert bool((x[1:] >= x[:-1]).all())
    nd = np.asarray(r.ndmpart_x, np.int64)
    assert nd[0] >= 0 and nd[-1] == n and (np.diff(nd) >= 0).all()
    # every particle counted in slab i lies below the slab's upper edge
    radx, dx = grid.malla(cfg.nx, np.float32(cfg.lado0))
    xs = x.cpu().numpy()
    for i in range(1, cfg.nx + 1, 37):
        if nd[i] > 0:
            assert xs[nd[i] - 1] <= np.float32(radx[i]) + np.float32(0.5) * np.float32(dx) + 1e-3
    # the store is a permutation of the input
    ids = torch.sort(out[7].long()).values
    assert bool((ids == torch.sort(snap.id.long()).values).all())


def test_catalogue_and_id_stream(run512):
    import torch
    cfg, snap, plan, b, r = run512
    cat = r.cat
    n = cat.nclus
    live = np.nonzero(cat.realclus[:n] != 0)[0]
    ind = cat.indcs[:n][live].astype(np.int64)
    lo, hi = ind[:, 0], ind[:, 1]
    assert (lo >= 1).all() and (hi >= lo - 1).all()
    order = np.argsort(lo, kind="stable")
    assert (lo[order][1:] > hi[order][:-1]).all()        # ranges do not overlap
    pph = r.pph
    assert hi.max() <= pph.shape[0]
    assert (cat.dmpclus[:n][live] >= plan.consts.min_num_part).all()
    rc = cat.realclus[:n][live]
    hal, sub = live[rc == -1], live[rc > 0]   # haloes; subhaloes (REALCLUS = host)
    assert hal.size > 100000 and sub.size > 1000
    assert (cat.masa[:n][hal] > 0).all() and (cat.radio[:n][hal] > 0).all()
    # a subhalo's mass and radius are MSUB and RSUB (MASA and RADIO stay 0
    # when its SO walk finds no virial crossing, as in the reference)
    assert (cat.msub[:n][sub] > 0).all() and (cat.rsub[:n][sub] > 0).all()
    assert (rc[rc > 0] <= n).all()
    half = cfg.lado0 / 2
    for f in ("clusrx", "clusry", "clusrz"):
        v = getattr(cat, f)[:n][live]
        assert (np.abs(v) <= half * 1.0001).all()
    # IDs valid and unique within each halo: sort (halo, id) keys on the device
    ids = pph.long() if hasattr(pph, "long") else torch.tensor(pph, device="cuda:0").long()
    idx = torch.arange(live.size, device="cuda:0", dtype=torch.long)
    starts = torch.tensor(lo - 1, device="cuda:0")
    lens = torch.tensor(hi - lo + 1, device="cuda:0")
    owner = torch.repeat_interleave(idx, lens)
    pos = torch.repeat_interleave(starts, lens) + (torch.arange(int(lens.sum()), device="cuda:0") -
                                                   torch.repeat_interleave(torch.cumsum(lens, 0) - lens, lens))
    vals = ids[pos]
    assert bool((vals >= 1).all()) and bool((vals <= snap.x.shape[0]).all())
    key = torch.sort(owner * (1 << 32) + vals).values
    assert bool((key[1:] != key[:-1]).all())


def test_window_matches_oracle(run512):
    import json
    import torch
    cfg, snap, plan, b, r = run512
    n = snap.x.shape[0]
    out = [torch.empty(n, dtype=torch.float32, device="cuda:0") for _ in range(7)] + \
          [torch.empty(n, dtype=torch.int32, device="cuda:0")]
    b.a.download_particles(out)
    torch.cuda.synchronize()
    store = W.OracleStore(*(t.cpu().numpy() for t in out), r.ndmpart_x)
    del out
    rng = np.random.default_rng(20261203)
    reports = []
    for call in b.calls:
        rows = W.choose_rows(call, rng)
        if rows.size == 0:
            continue
        ocat, opph, margins = W.run_oracle_rows(call, rows, store, plan.consts, plan.mesh)
        reports.append(W.compare_rows(call, rows, ocat, opph, margins))
    tot = {k: sum(rep["margins"][k] for rep in reports) for k in reports[0]["margins"]}
    summary = {"calls": len(reports), "rows": sum(rep["rows"] for rep in reports),
               "bound_ids": sum(rep["bound_ids"] for rep in reports),
               "largest_rows_members": int(max(int(c.post.dmpclus[c.low1 - 1:c.low2].max(initial=0))
                                               for c in b.calls)),
               "margins_1e-6": tot,
               "rows_with_margin": sum(rep["rows_with_margin"] for rep in reports),
               "explained_mismatches": {f"{rep['kind']}{rep['low1']}": rep["explained"] for rep in reports
                                        if rep["explained"]}}
    print("parity-512-window", json.dumps(summary))
    unexplained = {f"{rep['kind']}{rep['low1']}": rep["unexplained"] for rep in reports if rep["unexplained"]}
    assert not unexplained, unexplained
    assert summary["rows"] > 1000
