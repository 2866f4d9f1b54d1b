"""The window-parity harness (tests/window_parity.py) on the CPU: the
oracle run through the recorder, then rerun on windows of rows, must agree
with itself row for row, and a difference planted in the recorded oracle
result must be reported (as unexplained where the oracle counted no
decision within 1e-6 of its threshold in that row)."""
import numpy as np

from asohf_b200 import driver, synth
from oracle import oracle as O
from tests import window_parity as W


def _recorded(name="small"):
    s = synth.generate(name)
    plan = driver.prepare(s)
    ob = O.OracleBackend()
    rec = W.Recorder(ob)
    driver.execute(plan, rec, with_subs=True)
    p = ob.p
    store = W.OracleStore(p.x, p.y, p.z, p.vx, p.vy, p.vz, p.m, p.id, ob.ndmpart_x)
    return plan, rec, store


def test_window_rerun_equals_full_run():
    plan, rec, store = _recorded()
    assert any(c.kind == "halo" for c in rec.calls)
    rng = np.random.default_rng(3)
    checked = 0
    for call in rec.calls:
        rows = W.choose_rows(call, rng, n_random=5, n_largest=3)
        if rows.size == 0:
            continue
        ocat, opph, margins = W.run_oracle_rows(call, rows, store, plan.consts, plan.mesh)
        rep = W.compare_rows(call, rows, ocat, opph, margins)
        assert not rep["unexplained"] and not rep["explained"], rep
        checked += rows.size
    assert checked > 5


def test_planted_difference_is_reported():
    plan, rec, store = _recorded()
    call = next(c for c in rec.calls if c.kind == "halo" and (c.post.realclus[c.low1 - 1:c.low2] != 0).any())
    rows = W.choose_rows(call, np.random.default_rng(0), n_random=0, n_largest=2)
    ocat, opph, margins = W.run_oracle_rows(call, rows, store, plan.consts, plan.mesh)
    r = int(rows[0])
    margins.rows[r] = 0
    ocat.dmpclus[r] += 1            # planted in the oracle's result
    ocat.masa[r] *= np.float32(1.001)
    rep = W.compare_rows(call, rows, ocat, opph, margins)
    assert set(rep["unexplained"][r]) >= {"dmpclus", "masa"}
    margins.rows[r, 2] = 1          # a near-threshold escape-energy test in that row
    rep = W.compare_rows(call, rows, ocat, opph, margins)
    assert r in rep["explained"] and not rep["unexplained"]
