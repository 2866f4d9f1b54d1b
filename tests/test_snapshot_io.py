"""The reference's particle inputs: the generic file
(readers/particle_general.f: record layout, split records, the stellar block
and the unit conversion), GADGET format 2 (readers/gadget_unformatted.f) and
MASCLET outputs (readers/masclet.f: the list-directed grids file, level
order, masses, the sign fix of heavy particles, stars and black holes), and
pipeline runs from files equal to the run from memory."""
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


# ---------------------------------------------------------------- MASCLET
def masclet_levels(seed, sizes=(300, 120, 40), npatch=(0, 3, 5), heavy=False):
    """Dark matter per level: the base level's mass is MAP (the file holds no
    masses there), the refined levels' masses are their own."""
    rng = np.random.default_rng(seed)
    out = []
    for ir, n in enumerate(sizes):
        d = block(n, seed + ir)
        d["id"] = (rng.permutation(n) + 1 + 10000 * ir).astype(np.int32)
        if ir > 0:
            d["npatch"] = npatch[ir]
            d["m"] = np.full(n, np.float32(0.5 ** (ir + 1)), np.float32)
        out.append(d)
    return out


@pytest.mark.parametrize("heavy", [False, True])
def test_masclet_round_trip(tmp_path, heavy):
    """Level order, MAP as the base level's mass, the refined levels' own
    masses, and READ_PARTICLES_MASCLET's sign fix: when the heaviest mass is
    more than four times the lightest, every particle above 0.9 of it gets a
    negative ID (masclet.f:389-400)."""
    lv = masclet_levels(5)
    mp = 1.0 if heavy else 0.25  # levels 0.25, 0.125: only 1.0 is more than 4 x the lightest
    d = str(tmp_path / "simu_masclet")
    sio.write_masclet(d, 7, 0.5, 1.5, mp, lv)
    r = sio.read_masclet(d, 7)
    assert r.n == r.n_dm == 460 and r.n_st == 0 and r.zeta == np.float32(1.5) and r.t == np.float32(0.5)
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(getattr(r, k), np.concatenate([l[k] for l in lv]))
    m = np.concatenate([np.full(300, np.float32(mp), np.float32), lv[1]["m"], lv[2]["m"]])
    assert np.array_equal(r.m, m)
    ids = np.concatenate([l["id"] for l in lv])
    if heavy:
        big = m > np.float32(0.9) * m.max()
        assert big.sum() == 300
        ids = np.where(big, -np.abs(ids), ids)
    assert np.array_equal(r.id, ids)


def test_masclet_stars_and_black_holes(tmp_path):
    """VAR = 2: the stars follow the dark matter, level by level; base-level
    stars keep ID 0 (the reference reads no IDs there), the others are offset
    by the largest dark-matter ID; the black holes' records are skipped."""
    lv = masclet_levels(9, sizes=(200, 80, 30))
    st = [block(10, 50), block(6, 51), block(4, 52)]
    d = str(tmp_path / "m")
    sio.write_masclet(d, 3, 0.1, 0.0, 0.5, lv, stars=st, nbh=[0, 2, 3])
    r = sio.read_masclet(d, 3, var=2)
    assert r.n_dm == 310 and r.n_st == 20 and r.n == 330
    assert np.array_equal(r.x[310:], np.concatenate([s["x"] for s in st]))
    assert np.array_equal(r.m[310:], np.concatenate([s["m"] for s in st]))
    mx = int(r.id[:310].max())
    assert np.array_equal(r.id[310:320], np.zeros(10, np.int32))
    assert np.array_equal(r.id[320:], np.concatenate([st[1]["id"], st[2]["id"]]) + mx)
    # without VAR = 2 the stellar file is not read
    assert sio.read_masclet(d, 3).n == 310


def test_masclet_grids_list_directed(tmp_path):
    """The grids file is read the way Fortran's list-directed READ reads it:
    values may span lines and use D exponents; a bare READ skips one line."""
    d = tmp_path / "g"
    d.mkdir()
    (d / "grids00001").write_text(" 1, 2.5D-01\n 2 1.0D0\n 3.0E+00\n 0 10\n 2\n"
                                  " 1 2 5 0 0\n skipped\n" + " a\n b\n c\n d\n" * 2 +
                                  " 2 1\n 3 0 0\n skipped\n p\n q\n r\n s\n")
    g = sio._masclet_grids(str(d / "grids00001"))
    assert g.nl == 2 and g.t == np.float32(0.25) and g.map == np.float32(1.0) and g.zeta == np.float32(3.0)
    assert g.npart == [10, 5, 3] and g.npatch == [0, 2, 1] and g.npartst == [2, 0, 0]


def test_pipeline_from_a_masclet_output_equals_the_run_from_memory(tmp_path):
    from asohf_b200 import driver, synth
    from oracle import oracle as O
    s = synth.generate("tiny")
    lv = [{"x": s.x, "y": s.y, "z": s.z, "vx": s.vx, "vy": s.vy, "vz": s.vz, "id": s.id}]
    d = str(tmp_path / "simu_masclet")
    sio.write_masclet(d, 1, 0.0, 0.0, float(s.m[0]), lv)
    parts = sio.read_masclet(d, 1)
    assert np.array_equal(parts.m, s.m)
    plan = driver.prepare(s)
    a = driver.execute(plan, O.OracleBackend(nthreads=1), with_subs=False)
    b = driver.execute(plan, O.OracleBackend(nthreads=1), with_subs=False, particles=parts)
    n = a.cat.nclus
    assert np.array_equal(a.u1, b.u1)
    assert np.array_equal(a.cat.realclus[:n], b.cat.realclus[:n]) and np.array_equal(a.pph, b.pph)
