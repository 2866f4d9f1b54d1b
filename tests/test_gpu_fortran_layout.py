"""The library called from C the way the Fortran shim calls it
(tests/fortran_layout_driver.c): host arrays in the Fortran driver's
layouts -- U1(NMAX,NMAY,NMAZ), U11(32,32,32,NPALEV), NPATCH(0:NLEVELS),
NDMPART_X(0:NMAX), catalogue arrays of MAXNCLUS entries, particle arrays
longer than N_DM -- and the calls in asohf.f's order, RE_SORT_HALOES
included.  Its outputs must equal the CPU oracle's run of the same
snapshot (128^3 particles, the 512^3 benchmark recipe at 1/64 of the
volume, haloes and subhaloes over 6 levels) through the Python driver: species counts, slab table, base grid
and every integer catalogue field identical, the ID stream identical,
patch densities within 2e-7 and float catalogue fields within 1e-5
relative."""
import os
import subprocess
from types import SimpleNamespace

import numpy as np
import pytest

from asohf_b200 import abi, api, driver, synth
from oracle import oracle as O
from tests import window_parity as W
from tests.catalogue_compare import compare

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NLEVELS = 9


def _write_input(path, plan, subs, n_extra=64):
    s, cfg = plan.snap, plan.snap.cfg
    k, cos, mesh, cand = plan.consts, plan.cos, plan.mesh, plan.cand
    n = s.x.shape[0]
    nl = mesh.nl
    nsub_lev = np.zeros(nl + 1, np.int32)
    sub_cols = {f: [] for f in ("clusrx", "clusry", "clusrz", "rsub", "realclus", "levhal")}
    for c in subs:
        nsub_lev[c.ir] = c.low2 - c.low1 + 1
        for f in sub_cols:
            sub_cols[f].append(getattr(c.pre, f)[c.low1 - 1:c.low2])
    sub_cols = {f: (np.concatenate(v) if v else np.zeros(0)) for f, v in sub_cols.items()}
    nsub = int(nsub_lev.sum())
    ncand = int(cand.clusrx.shape[0])
    cap = ncand + nsub + 1000
    h = np.zeros(16, np.int64)
    h[:14] = [n, cfg.nx, nl, mesh.total, cap, ncand, nsub, 2, k.min_num_part, k.do_compute_energies,
              k.max_part_dsum, k.flag_wdm, k.var, n + n_extra]
    fh = np.zeros(16, np.float32)
    fh[:14] = [cfg.lado0, plan.dx, cos["rodo"], cos["re0"], k.rote, k.rete, k.pi, k.cgr, k.um, k.uv,
               k.contrastec, k.omegaz, k.fdm, k.zeta]
    npatch = np.zeros(NLEVELS + 1, np.int32)
    npatch[: nl + 1] = mesh.npatch[: nl + 1]
    f32 = lambda a: np.ascontiguousarray(a, np.float32)
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    with open(path, "wb") as f:
        for a in (h, fh, f32(s.x), f32(s.y), f32(s.z), f32(s.vx), f32(s.vy), f32(s.vz), f32(s.m), i32(s.id),
                  npatch, i32(mesh.patchnx), i32(mesh.patchny), i32(mesh.patchnz), i32(mesh.patchx),
                  i32(mesh.patchy), i32(mesh.patchz), f32(mesh.patchrx), f32(mesh.patchry),
                  f32(mesh.patchrz), i32(mesh.pare), i32(cand.nhallev[: nl + 1]),
                  f32(cand.clusrx), f32(cand.clusry), f32(cand.clusrz), f32(cand.radio), f32(cand.masa),
                  i32(cand.levhal), i32(cand.patchclus), i32(nsub_lev),
                  f32(sub_cols["clusrx"]), f32(sub_cols["clusry"]), f32(sub_cols["clusrz"]),
                  f32(sub_cols["rsub"]), i32(sub_cols["realclus"]), i32(sub_cols["levhal"])):
            a.tofile(f)


def _read_output(path, nx, npt):
    buf = open(path, "rb").read()
    off = 0

    def take(dt, cnt):
        nonlocal off
        a = np.frombuffer(buf, dt, cnt, off)
        off += a.nbytes
        return a.copy()

    out = SimpleNamespace()
    out.npart_esp = take(np.int32, abi.N_ESP)
    out.u1 = take(np.float32, nx ** 3)
    out.u11 = take(np.float32, npt * abi.NAMRX ** 3).reshape(npt, -1)
    out.ndmpart_x = take(np.int32, nx + 1)
    nclus = int(take(np.int64, 1)[0])
    cat = abi.Catalogue(max(nclus, 1))
    cat.nclus = nclus
    for f in abi.CAT_SCALAR_FLOAT:
        getattr(cat, f)[:nclus] = take(np.float32, nclus)
    for f in abi.CAT_SCALAR_INT:
        getattr(cat, f)[:nclus] = take(np.int32, nclus)
    for f, w in abi.CAT_MULTI.items():
        dt = np.int32 if f == "indcs" else np.float32
        getattr(cat, f)[:nclus] = take(dt, nclus * w).reshape(nclus, w)
    out.cat = cat
    out.subs_lev = take(np.int32, NLEVELS + 1)
    npph = int(take(np.int64, 1)[0])
    out.pph = take(np.int32, npph)
    assert off == len(buf)
    return out


def test_fortran_layout_driver_matches_oracle(gpu_lib, tmp_path):
    s = synth.generate("cfg4s")
    plan = driver.prepare(s)
    rec = W.Recorder(O.OracleBackend())
    ro = driver.execute(plan, rec, with_subs=True)
    subs = [c for c in rec.calls if c.kind == "sub"]
    assert subs, "the workload must exercise SUBSTRUCTURE_PARTICLES"
    exe = str(tmp_path / "fortran_layout_driver")
    libdir = os.path.dirname(api.lib_path())
    subprocess.run(["gcc", "-std=c11", "-O1", "-Wall", os.path.join(ROOT, "tests", "fortran_layout_driver.c"),
                    "-I", os.path.join(ROOT, "include"), "-L", libdir, "-lasohf_gpu",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True)
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    _write_input(fin, plan, subs)
    r = subprocess.run([exe, fin, fout], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = _read_output(fout, s.cfg.nx, plan.mesh.total)
    assert np.array_equal(c.npart_esp, ro.npart_esp)
    assert np.array_equal(c.ndmpart_x, ro.ndmpart_x)
    assert np.array_equal(c.u1, np.asarray(ro.u1).reshape(-1))
    if plan.mesh.total:
        assert np.allclose(c.u11, np.asarray(ro.u11), rtol=2e-7, atol=0)
    assert np.array_equal(c.subs_lev[: plan.mesh.nl + 1], ro.subs_lev)
    live = ro.cat.realclus[: ro.cat.nclus] != 0
    assert live.sum() > 10 and (ro.cat.realclus[: ro.cat.nclus] > 0).any()
    # the stream up to the last live halo's range, as the driver returns it
    n_ids = int(ro.cat.indcs[: ro.cat.nclus][live][:, 1].max())
    assert c.pph.shape[0] >= n_ids
    compare(SimpleNamespace(cat=c.cat, pph=c.pph[:n_ids]), ro)
