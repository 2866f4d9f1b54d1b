"""The reference's catalogue outputs (asohf.f:800-910): FORMAT 112 edit
descriptors, FRACTION_MASS_SUBS, and round trips of the families and
particles files."""
import numpy as np
import pytest

from asohf_b200 import abi, catalogue_io as cio


def test_edit_descriptors():
    assert cio.fmt_e(12345.6, 14, 6) == "  0.123456E+05"
    assert cio.fmt_e(-0.000123456, 14, 6) == " -0.123456E-03"
    assert cio.fmt_e(0.0, 14, 6) == "  0.000000E+00"
    assert cio.fmt_e(99999.996, 14, 6) == "  0.100000E+06"      # the carry moves the exponent
    assert cio.fmt_e(1.5e12, 14, 3) == "     0.150E+13"
    assert cio.fmt_f(3.14159265, 14, 6) == "      3.141593"
    assert cio.fmt_f(-1e-7, 14, 6) == "     -0.000000"
    assert cio.fmt_f(1e12, 14, 6) == "*" * 14                 # does not fit
    assert cio.fmt_f(-12.5, 14, 3) == "       -12.500"
    assert cio.fmt_i(12, 14) == " " * 12 + "12" and cio.fmt_i(-3, 14) == " " * 12 + "-3"
    assert len(cio.parse_format(cio.FORMAT_112)) == 51 == len(cio.HEADER_1) == len(cio.HEADER_2)
    with pytest.raises(ValueError):
        cio.format_record([1, 2, 3])


def small_catalogue():
    c = abi.Catalogue(8)
    c.nclus = 5
    c.realclus[:5] = [-1, 1, 1, 2, 0]        # host, two subhaloes of it, one of the first subhalo, one removed
    c.masa[:5] = [10.0, 0, 0, 0, 4.0]
    c.msub[:5] = [0, 1.0, 2.0, 0.5, 0]
    return c


def test_fraction_mass_subs():
    fsub, nsubs = cio.fraction_mass_subs(small_catalogue())
    assert list(nsubs) == [2, 1, 0, 0, 0]
    assert np.allclose(fsub, [0.3, 0.5, 0.0, 0.0, 0.0])
    assert fsub.dtype == np.float32


def random_catalogue(n, seed):
    rng = np.random.default_rng(seed)
    c = abi.Catalogue(n + 2)
    c.nclus = n
    c.realclus[:n] = np.where(rng.random(n) < 0.8, -1, 0)
    for f in ("clusrx", "clusry", "clusrz", "clusrxcm", "clusrycm", "clusrzcm"):
        getattr(c, f)[:n] = rng.uniform(-50, 50, n)
    c.masa[:n] = 10 ** rng.uniform(10, 15, n)
    c.radio[:n] = rng.uniform(0.05, 2.0, n)
    c.dmpclus[:n] = rng.integers(20, 100000, n)
    c.iplip[:n] = rng.integers(1, 10 ** 7, n)
    c.vx[:n], c.vy[:n], c.vz[:n] = rng.normal(0, 1e-3, (3, n))
    c.eigenval[:n] = rng.uniform(0.01, 1.0, (n, 3))
    c.m200c[:n] = c.masa[:n] * 0.9
    c.r200c[:n] = c.radio[:n] * 0.8
    sizes = c.dmpclus[:n].astype(np.int64)
    ends = np.cumsum(sizes)
    c.indcs[:n, 0] = ends - sizes + 1
    c.indcs[:n, 1] = ends
    return c, int(ends[-1])


def test_families_round_trip(tmp_path):
    c, _ = random_catalogue(40, 1)
    uv = 299792.46
    p = tmp_path / "families00001"
    nkeep = cio.write_families(str(p), c, 1, 0.0, uv)
    rows = cio.read_families(str(p))
    keep = np.nonzero(c.realclus[:40] != 0)[0]
    assert rows.shape == (nkeep, 51) and nkeep == len(keep)
    assert np.array_equal(rows[:, 0], keep + 1)
    assert np.allclose(rows[:, 2], c.clusrx[keep], atol=5e-7)                 # F14.6
    assert np.allclose(rows[:, 5], c.masa[keep], rtol=5e-6)                   # E14.6
    assert np.array_equal(rows[:, 9], c.dmpclus[keep])                        # I14
    assert np.allclose(rows[:, 27], (c.vx[keep] * np.float32(uv)).astype(np.float32), atol=5e-4)  # F14.3
    lines = p.read_text().splitlines()
    assert all(len(ln) == 14 * 51 for ln in lines[7:])


def test_particles_round_trip(tmp_path):
    c, total = random_catalogue(30, 2)
    pph = np.arange(1, total + 1, dtype=np.int32)[::-1].copy()
    p = tmp_path / "particles00001"
    cio.write_particles(str(p), c, pph)
    r = cio.read_particles(str(p))
    keep = np.nonzero(c.realclus[:30] != 0)[0]
    assert [h[0] for h in r["haloes"]] == list(keep + 1)
    assert all((h[1], h[2]) == tuple(c.indcs[i]) for h, i in zip(r["haloes"], keep))
    last = max(c.indcs[i, 1] for i in keep)
    assert np.array_equal(r["ids"], pph[:last])


def test_write_outputs_names_and_pipeline(tmp_path):
    """The driver's result on the 32^3 test snapshot (oracle backend) goes
    out as families00007 / particles00007, and the ID stream reads back."""
    from asohf_b200 import driver, synth
    from oracle import oracle as O
    r = driver.run(synth.generate("tiny"), O.OracleBackend(nthreads=1), with_subs=True)
    paths = cio.write_outputs(str(tmp_path), 7, r.cat, r.pph, 0.0, 299792.46)
    assert [p.split("/")[-1] for p in paths] == ["families00007", "particles00007"]
    back = cio.read_particles(paths[1])
    n = r.cat.nclus
    assert len(back["haloes"]) == int((r.cat.realclus[:n] != 0).sum())
    assert np.array_equal(back["ids"], np.asarray(r.pph)[:back["ids"].shape[0]])
    rows = cio.read_families(paths[0])
    assert rows.shape[0] == len(back["haloes"])
