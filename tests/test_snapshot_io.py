"""The reference's generic particle input (readers/particle_general.f):
record layout, split records, the stellar block and the unit conversion,
and a pipeline run from a file equal to the run from memory."""
import io

import numpy as np
import pytest

from asohf_b200 import snapshot_io as sio


def block(n, seed):
    rng = np.random.default_rng(seed)
    d = {k: rng.normal(0, 10, n).astype(np.float32) for k in sio.FIELDS}
    d["m"] = np.abs(d["m"]) + 1
    d["id"] = rng.permutation(n).astype(np.int32) + 1
    return d


def test_split_records_round_trip():
    payload = bytes(range(256)) * 3
    f = io.BytesIO()
    sio.write_record(f, payload, max_sub=100)
    sio.write_record(f, b"tail", max_sub=100)
    f.seek(0)
    assert sio.read_record(f) == payload and sio.read_record(f) == b"tail" and sio.read_record(f) is None
    f = io.BytesIO(f.getvalue()[:-3])
    sio.read_record(f)
    with pytest.raises(ValueError):
        sio.read_record(f)


def test_generic_file_round_trip_and_units(tmp_path):
    dm, st = block(500, 1), block(70, 2)
    p = str(tmp_path / "particles00001")
    sio.write_particles_general(p, 1.5, dm, st, max_sub=1000)
    r = sio.read_particles_general(p, var=2, cio_mass=2.0, cio_speed=3.0, cio_length=0.5, cio_alpha=1.0,
                                   cio_xc=1.0, cio_yc=-2.0, cio_zc=0.25, um=4.0, uv=6.0)
    assert (r.n_dm, r.n_st, r.n) == (500, 70, 570) and r.zeta == 1.5
    x = np.concatenate([dm["x"], st["x"]])
    assert np.array_equal(r.x, ((x - np.float32(1.0)) * np.float32(0.5)).astype(np.float32))
    assert np.array_equal(r.vx, np.concatenate([dm["vx"], st["vx"]]) * np.float32(0.5))   # 3/6, alpha = 1
    assert np.array_equal(r.m, np.concatenate([dm["m"], st["m"]]) * np.float32(0.5))      # 2/4
    assert np.array_equal(r.id, np.concatenate([dm["id"], st["id"]]))
    r1 = sio.read_particles_general(p, var=1)
    assert r1.n == 500 and r1.n_st == 0


def test_pipeline_from_a_file_equals_the_run_from_memory(tmp_path):
    from asohf_b200 import driver, synth
    from oracle import oracle as O
    s = synth.generate("tiny")
    p = str(tmp_path / "particles00001")
    sio.write_particles_general(p, 0.0, {"x": s.x, "y": s.y, "z": s.z, "vx": s.vx, "vy": s.vy, "vz": s.vz,
                                         "m": s.m, "id": s.id})
    parts = sio.read_particles_general(p)
    plan = driver.prepare(s)
    a = driver.execute(plan, O.OracleBackend(nthreads=1), with_subs=False)
    b = driver.execute(plan, O.OracleBackend(nthreads=1), with_subs=False, particles=parts)
    n = a.cat.nclus
    assert np.array_equal(a.u1, b.u1)
    assert np.array_equal(a.cat.realclus[:n], b.cat.realclus[:n]) and np.array_equal(a.pph, b.pph)


def gadget_case(npp, header_dm_mass, seed):
    rng = np.random.default_rng(seed)
    ntot = sum(npp)
    pos = rng.uniform(0, 100, (ntot, 3)).astype(np.float32)
    vel = rng.normal(0, 300, (ntot, 3)).astype(np.float32)
    ids = rng.permutation(ntot).astype(np.int32) + 1000
    m_all = rng.uniform(1, 2, ntot).astype(np.float32)
    mass_arr = [0.0] * 6
    if header_dm_mass:
        mass_arr[1] = 0.75
        keep = np.r_[0:npp[0], sum(npp[:4]):ntot]   # the block skips types 1-3
        masses = m_all[keep]
    else:
        masses = m_all
    return pos, vel, ids, m_all, mass_arr, masses


@pytest.mark.parametrize("header_dm_mass", [True, False])
def test_gadget_format2(tmp_path, header_dm_mass):
    npp = [30, 200, 10, 5, 40, 2]          # gas, dm (three types), stars, black holes
    pos, vel, ids, m_all, mass_arr, masses = gadget_case(npp, header_dm_mass, 3)
    p = str(tmp_path / "snap_001")
    sio.write_gadget_format2(p, npp, mass_arr, 0.5, pos, vel, ids, masses, boxsize=100.0)
    r = sio.read_gadget_unformatted(p, var=2, cio_length=0.5, cio_xc=50.0, cio_yc=50.0, cio_zc=50.0)
    dm = slice(30, 245)
    st = slice(245, 285)
    assert (r.n_dm, r.n_st, r.n) == (215, 40, 255) and r.zeta == 0.5
    assert np.array_equal(r.x[:215], ((pos[dm, 0] - np.float32(50)) * np.float32(0.5)).astype(np.float32))
    assert np.array_equal(r.vz[215:], vel[st, 2])
    assert np.array_equal(r.id, np.r_[31:246, 246:286].astype(np.int32))    # numbered by file position
    if header_dm_mass:
        assert (r.m[:215] == np.float32(0.75)).all()
    else:
        assert np.array_equal(r.m[:215], m_all[dm])
    assert np.array_equal(r.m[215:], m_all[st])
    r1 = sio.read_gadget_unformatted(p, var=1)
    assert r1.n == 215 and r1.n_st == 0
