"""Particle input in the reference's formats: the generic file
(readers/particle_general.f), GADGET format-2 snapshots
(readers/gadget_unformatted.f) and MASCLET outputs (readers/masclet.f).

The generic file (readers/particle_general.f) is a
Fortran unformatted sequential file `simulation/particlesNNNNN` holding
ZETA; N_DM; the x, y, z, vx, vy, vz, mass arrays (REAL*4) and the IDs
(INTEGER*4) of the dark-matter particles; and, when VAR = 2, N_ST and the
same eight arrays for the stars.  After reading, the reference converts
units in REAL*4 (particle_general.f:141-161): positions (x - CIO_XC) *
CIO_LENGTH, velocities * (CIO_SPEED / UV) * (1 + ZETA)**(CIO_ALPHA - 1),
masses * CIO_MASS / UM.

Records use gfortran's layout: a 4-byte length before and after each
record; a record longer than 2**31 - 9 bytes is split into subrecords whose
leading marker is negative while more follow (and whose trailing marker is
negative on all but the first).
"""
from __future__ import annotations

import struct
from types import SimpleNamespace

import numpy as np

MAX_SUBRECORD = 2 ** 31 - 9


def write_record(f, payload: bytes, max_sub: int = MAX_SUBRECORD) -> None:
    """One Fortran unformatted sequential record (split into subrecords)."""
    n = len(payload)
    if n <= max_sub:
        f.write(struct.pack("<i", n) + payload + struct.pack("<i", n))
        return
    off, first = 0, True
    while off < n:
        k = min(max_sub, n - off)
        more = off + k < n
        f.write(struct.pack("<i", -k if more else k))
        f.write(payload[off:off + k])
        f.write(struct.pack("<i", k if first else -k))
        off += k
        first = False


def read_record(f) -> bytes | None:
    """The next record (its subrecords joined); None at the end of the file."""
    parts = []
    while True:
        h = f.read(4)
        if not h:
            if parts:
                raise ValueError("file ends inside a record")
            return None
        (lead,) = struct.unpack("<i", h)
        k = abs(lead)
        body = f.read(k)
        t = f.read(4)
        if len(body) != k or len(t) != 4 or abs(struct.unpack("<i", t)[0]) != k:
            raise ValueError("broken record marker")
        parts.append(body)
        if lead >= 0:
            return b"".join(parts)


FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m")


def write_particles_general(path: str, zeta: float, dm: dict, stars: dict | None = None,
                            max_sub: int = MAX_SUBRECORD) -> None:
    """Writes the generic input file; dm / stars hold x..m (float32) and id
    (int32) arrays in the file's own units."""
    with open(path, "wb") as f:
        write_record(f, struct.pack("<f", np.float32(zeta)), max_sub)
        for blk in ([dm] + ([stars] if stars is not None else [])):
            n = int(np.asarray(blk["x"]).shape[0])
            write_record(f, struct.pack("<i", n), max_sub)
            for k in FIELDS:
                write_record(f, np.ascontiguousarray(blk[k], np.float32).tobytes(), max_sub)
            write_record(f, np.ascontiguousarray(blk["id"], np.int32).tobytes(), max_sub)


def read_particles_general(path: str, var: int = 1, cio_mass: float = 1.0, cio_speed: float = 1.0,
                           cio_length: float = 1.0, cio_alpha: float = 1.0, cio_xc: float = 0.0,
                           cio_yc: float = 0.0, cio_zc: float = 0.0, um: float = 1.0,
                           uv: float = 1.0) -> SimpleNamespace:
    """READ_PARTICLES_GENERAL (readers/particle_general.f:2-178): the
    particles (dark matter first, then stars when var = 2) in internal
    units, as float32/int32 arrays ready for the device upload, with zeta,
    n_dm and n_st."""
    with open(path, "rb") as f:
        (zeta,) = struct.unpack("<f", read_record(f))
        blocks = []
        for _ in range(2 if var == 2 else 1):
            (n,) = struct.unpack("<i", read_record(f))
            arr = {}
            for k in FIELDS:
                a = np.frombuffer(read_record(f), np.float32)
                if a.shape[0] != n:
                    raise ValueError(f"{k}: {a.shape[0]} values for {n} particles")
                arr[k] = a
            ids = np.frombuffer(read_record(f), np.int32)
            if ids.shape[0] != n:
                raise ValueError(f"id: {ids.shape[0]} values for {n} particles")
            arr["id"] = ids
            blocks.append(arr)
    f32 = np.float32
    fact_mass = f32(f32(cio_mass) / f32(um))
    fact_speed = f32(f32(f32(cio_speed) / f32(uv)) * f32(np.power(f32(1.0) + f32(zeta), f32(f32(cio_alpha) - f32(1.0)),
                                                                 dtype=np.float32)))
    fact_length = f32(cio_length)
    cat = {k: np.concatenate([b[k] for b in blocks]) for k in FIELDS + ("id",)}
    out = SimpleNamespace(zeta=float(zeta), n_dm=int(blocks[0]["x"].shape[0]),
                          n_st=int(blocks[1]["x"].shape[0]) if len(blocks) > 1 else 0)
    for k, c in (("x", cio_xc), ("y", cio_yc), ("z", cio_zc)):
        setattr(out, k, ((cat[k] - f32(c)) * fact_length).astype(np.float32))
    for k in ("vx", "vy", "vz"):
        setattr(out, k, (cat[k] * fact_speed).astype(np.float32))
    out.m = (cat["m"] * fact_mass).astype(np.float32)
    out.id = cat["id"].astype(np.int32)
    out.n = out.x.shape[0]
    return out


def write_gadget_format2(path: str, npp, mass_arr, zeta: float, pos, vel, ids, masses,
                         boxsize: float = 0.0, omega_m: float = 0.3, omega_l: float = 0.7, h: float = 0.7) -> None:
    """A GADGET format-2 snapshot (label records "HEAD", "POS ", "VEL ",
    "ID  ", "MASS" before each block) in the layout the reference's reader
    expects; pos/vel (ntot, 3) float32, ids int32, masses float32 for the
    types whose mass_arr entry is 0."""
    def label(f, name, nbytes):
        write_record(f, name.encode().ljust(4)[:4] + struct.pack("<i", nbytes + 8))
    head = (struct.pack("<6i", *npp) + struct.pack("<6d", *mass_arr) + struct.pack("<2d", 1.0 / (1.0 + zeta), zeta)
            + bytes(40) + struct.pack("<4d", boxsize, omega_m, omega_l, h))
    head = head.ljust(256, b"\0")
    with open(path, "wb") as f:
        for name, payload in (("HEAD", head), ("POS ", np.ascontiguousarray(pos, np.float32).tobytes()),
                              ("VEL ", np.ascontiguousarray(vel, np.float32).tobytes()),
                              ("ID  ", np.ascontiguousarray(ids, np.int32).tobytes()),
                              ("MASS", np.ascontiguousarray(masses, np.float32).tobytes())):
            label(f, name, len(payload))
            write_record(f, payload)


def read_gadget_unformatted(path: str, var: int = 1, cio_mass: float = 1.0, cio_speed: float = 1.0,
                            cio_length: float = 1.0, cio_alpha: float = 1.0, cio_xc: float = 0.0,
                            cio_yc: float = 0.0, cio_zc: float = 0.0, um: float = 1.0,
                            uv: float = 1.0) -> SimpleNamespace:
    """READ_GADGET_UNFORMATTED (readers/gadget_unformatted.f:2-278): a GADGET
    format-2 snapshot.  Dark matter is types 1-3 (NPP(2:4)), stars type 4
    (NPP(5), with var = 2); IDs are not read but numbered by position in the
    file, as the reference does; dark-matter masses come from the header's
    MASS_ARR(2) when it is positive (the mass block then holds every other
    particle), else from the mass block.  Units as in
    read_particles_general."""
    with open(path, "rb") as f:
        read_record(f)  # "HEAD" label
        hd = read_record(f)
        npp = struct.unpack("<6i", hd[:24])
        mass_arr = struct.unpack("<6d", hd[24:72])
        zeta = struct.unpack("<d", hd[80:88])[0]
        ntot = sum(npp)
        idm0, idm1 = npp[0], sum(npp[:4])            # 0-based [idm0, idm1)
        ist0, ist1 = idm1, sum(npp[:5])
        n_dm = idm1 - idm0
        n_st = ist1 - ist0 if var == 2 else 0
        read_record(f)
        pos = np.frombuffer(read_record(f), np.float32).reshape(ntot, 3)
        read_record(f)
        vel = np.frombuffer(read_record(f), np.float32).reshape(ntot, 3)
        read_record(f)
        read_record(f)  # the IDs: numbered instead (gadget_unformatted.f:165-172)
        lab = read_record(f)
        mrec = read_record(f) if lab is not None else b""
    mblock = np.frombuffer(mrec or b"", np.float32)
    if mass_arr[1] > 0.0:
        m_dm = np.full(n_dm, np.float32(mass_arr[1]), np.float32)
        st0m = npp[0]                               # the block skips the dark matter
    else:
        m_dm = mblock[idm0:idm1]
        st0m = ist0
    sel = [slice(idm0, idm1)] + ([slice(ist0, ist1)] if var == 2 else [])
    raw = SimpleNamespace(zeta=float(np.float32(zeta)))
    raw.x, raw.y, raw.z = (np.concatenate([pos[s, a] for s in sel]) for a in range(3))
    raw.vx, raw.vy, raw.vz = (np.concatenate([vel[s, a] for s in sel]) for a in range(3))
    masses = [m_dm] + ([mblock[st0m:st0m + n_st]] if var == 2 else [])
    raw.m = np.concatenate(masses).astype(np.float32)
    raw.id = np.concatenate([np.arange(s.start + 1, s.stop + 1, dtype=np.int32) for s in sel])
    f32 = np.float32
    fact_mass = f32(f32(cio_mass) / f32(um))
    fact_speed = f32(f32(f32(cio_speed) / f32(uv)) * np.power(f32(1.0) + f32(raw.zeta), f32(f32(cio_alpha) - f32(1.0)),
                                                              dtype=np.float32))
    fact_length = f32(cio_length)
    out = SimpleNamespace(zeta=raw.zeta, n_dm=n_dm, n_st=n_st, id=raw.id)
    for k, c in (("x", cio_xc), ("y", cio_yc), ("z", cio_zc)):
        setattr(out, k, ((getattr(raw, k) - f32(c)) * fact_length).astype(np.float32))
    for k in ("vx", "vy", "vz"):
        setattr(out, k, (getattr(raw, k) * fact_speed).astype(np.float32))
    out.m = (raw.m * fact_mass).astype(np.float32)
    out.n = out.x.shape[0]
    return out


# ---------------------------------------------------------------- MASCLET
# READ_PARTICLES_MASCLET (readers/masclet.f:241-525): a MASCLET output
# `simu_masclet/{grids,cldm,clst}NNNNN`.  `grids` is list-directed text:
# "IRR T NL MAP", "ZETA", "IR NDXYZ NST0", then per level IR = 1..NL the
# line "IRR NPATCH NPART NPARTST NPARTBH", one line the reader skips and four
# lines per patch it skips.  `cldm` is unformatted: a header record, the base
# density record, then X, Y, Z, VX, VY, VZ (REAL*4) and the IDs (INTEGER*4) of
# the NDXYZ base-level particles, whose mass is MAP; then per level one
# record per patch (its density, skipped) and X..VZ, the masses and the IDs
# of the level's NPART particles.  No unit conversion: MASCLET's units are
# the code's.  When the heaviest mass exceeds four times the lightest, the
# particles above 0.9 of the heaviest get a negative ID.  With VAR = 2 the
# stars come from `clst` (base level: NPARTST(0) + NPARTBH(0) particles,
# X..mass, two skipped records, no IDs, so their ID stays 0; each level:
# the patch records, X..mass of NPARTST(IR), two skipped records and IDs
# that are offset by the largest dark-matter ID; the black holes' nine
# records are skipped, as the reference does with CONSIDER_BH = 0).


def _masclet_grids(path: str):
    """The header and per-level counts of a MASCLET `grids` file, read with
    list-directed semantics (values may span lines; a bare READ skips one
    line)."""
    with open(path) as f:
        lines = f.read().splitlines()
    pos = [0]

    def values(n):
        out = []
        while len(out) < n:
            if pos[0] >= len(lines):
                raise ValueError(f"{path}: ends before {n} values")
            toks = lines[pos[0]].replace(",", " ").replace("d", "e").replace("D", "E").split()
            pos[0] += 1
            out += toks
        return out[:n]

    def skip():
        pos[0] += 1

    irr, t, nl, mp = values(4)
    (zeta,) = values(1)
    _, ndxyz, nst0 = values(3)
    nl = int(nl)
    npatch, npart, npartst, npartbh = [0], [int(ndxyz)], [int(nst0)], [0]
    for ir in range(1, nl + 1):
        v = values(5)
        npatch.append(int(v[1]))
        npart.append(int(v[2]))
        npartst.append(int(v[3]))
        npartbh.append(int(v[4]))
        skip()
        for _ in range(4 * npatch[ir]):
            skip()
    return SimpleNamespace(t=float(np.float32(float(t))), nl=nl, map=np.float32(float(mp)),
                           zeta=float(np.float32(float(zeta))), npatch=npatch, npart=npart,
                           npartst=npartst, npartbh=npartbh)


def _first(rec: bytes | None, dtype, n: int, what: str):
    if rec is None:
        raise ValueError(f"{what}: the file ends early")
    a = np.frombuffer(rec, dtype)
    if a.shape[0] < n:  # a longer record is read in part, as Fortran does
        raise ValueError(f"{what}: {a.shape[0]} values for {n} particles")
    return a[:n]


def read_masclet(directory: str, it: int, var: int = 1) -> SimpleNamespace:
    """READ_PARTICLES_MASCLET (readers/masclet.f:241-525) on the files of
    output `it` in `directory` (the reference's ./simu_masclet): the
    particles (dark matter level by level, then stars when var = 2) as
    float32/int32 arrays, with t, zeta, n_dm and n_st."""
    import os
    tag = "%05d" % it
    g = _masclet_grids(os.path.join(directory, "grids" + tag))
    cols = {k: [] for k in FIELDS + ("id",)}
    with open(os.path.join(directory, "cldm" + tag), "rb") as f:
        read_record(f)  # header
        read_record(f)  # base-level density
        n0 = g.npart[0]
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            cols[k].append(_first(read_record(f), np.float32, n0, "cldm " + k))
        cols["id"].append(_first(read_record(f), np.int32, n0, "cldm id"))
        cols["m"].append(np.full(n0, g.map, np.float32))
        for ir in range(1, g.nl + 1):
            for _ in range(g.npatch[ir]):
                read_record(f)  # patch density
            n = g.npart[ir]
            for k in FIELDS:
                cols[k].append(_first(read_record(f), np.float32, n, f"cldm level {ir} {k}"))
            cols["id"].append(_first(read_record(f), np.int32, n, f"cldm level {ir} id"))
    dm = {k: np.concatenate(v) if v else np.zeros(0) for k, v in cols.items()}
    dm["id"] = dm["id"].astype(np.int32)
    n_dm = int(dm["x"].shape[0])
    if n_dm:  # heavier species: negative IDs (masclet.f:389-400)
        mx = np.float32(dm["m"].max())
        if mx > np.float32(4.0) * np.float32(dm["m"].min()):
            bas = np.float32(np.float32(0.9) * mx)
            heavy = dm["m"] > bas
            dm["id"][heavy] = -np.abs(dm["id"][heavy])
    st = {k: [] for k in FIELDS + ("id",)}
    if var == 2:
        max_id = int(dm["id"].max()) if n_dm else 0
        with open(os.path.join(directory, "clst" + tag), "rb") as f:
            read_record(f)  # header
            read_record(f)  # base-level stellar density
            nb = g.npartst[0] + g.npartbh[0]
            for k in FIELDS:
                st[k].append(_first(read_record(f), np.float32, nb, "clst " + k))
            read_record(f)
            read_record(f)
            st["id"].append(np.zeros(nb, np.int32))  # not read at the base level
            for ir in range(1, g.nl + 1):
                for _ in range(g.npatch[ir]):
                    read_record(f)
                nb = g.npartst[ir]
                for k in FIELDS:
                    st[k].append(_first(read_record(f), np.float32, nb, f"clst level {ir} {k}"))
                read_record(f)
                read_record(f)
                ids = _first(read_record(f), np.int32, nb, f"clst level {ir} id")
                st["id"].append((ids.astype(np.int64) + max_id).astype(np.int32))
                for _ in range(9):  # black holes, not considered
                    read_record(f)
    stars = {k: np.concatenate(v) if v else np.zeros(0, np.int32 if k == "id" else np.float32)
             for k, v in st.items()}
    out = SimpleNamespace(t=g.t, zeta=g.zeta, n_dm=n_dm, n_st=int(stars["x"].shape[0]))
    for k in FIELDS:
        setattr(out, k, np.concatenate([dm[k], stars[k]]).astype(np.float32))
    out.id = np.concatenate([dm["id"], stars["id"]]).astype(np.int32)
    out.n = out.x.shape[0]
    return out


def write_masclet(directory: str, it: int, t: float, zeta: float, mp: float, levels: list,
                  stars: list | None = None, nbh: list | None = None) -> None:
    """Writes a MASCLET output in the layout read_masclet reads.  levels[ir]
    holds the dark matter of level ir (x..vz and id; m too for ir >= 1) and,
    for ir >= 1, npatch; stars[ir] (x..m, and id for ir >= 1) the stars; nbh
    the black-hole counts per level (their records hold zeros).  The grid
    records (densities, patch geometry) hold placeholders: the reader skips
    them."""
    import os
    os.makedirs(directory, exist_ok=True)
    tag = "%05d" % it
    nl = len(levels) - 1
    nbh = nbh if nbh is not None else [0] * (nl + 1)
    sts = stars if stars is not None else [None] * (nl + 1)
    nst = [0 if s is None else int(np.asarray(s["x"]).shape[0]) for s in sts]
    npatch = [0] + [int(levels[ir]["npatch"]) for ir in range(1, nl + 1)]
    with open(os.path.join(directory, "grids" + tag), "w") as f:
        f.write(f" {it} {t!r} {nl} {float(np.float32(mp))!r}\n {zeta!r}\n")
        f.write(f" 0 {int(np.asarray(levels[0]['x']).shape[0])} {nst[0]}\n")
        for ir in range(1, nl + 1):
            f.write(f" {ir} {npatch[ir]} {int(np.asarray(levels[ir]['x']).shape[0])} {nst[ir]} {nbh[ir]}\n")
            f.write(" ------\n")
            for p in range(npatch[ir]):
                f.write(" 8 8 8\n 1 1 1\n 0.0 0.0 0.0\n 0\n")
    dens = np.zeros(8, np.float32).tobytes()
    with open(os.path.join(directory, "cldm" + tag), "wb") as f:
        write_record(f, struct.pack("<ifff", it, t, 0.0, zeta))
        write_record(f, dens)
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            write_record(f, np.ascontiguousarray(levels[0][k], np.float32).tobytes())
        write_record(f, np.ascontiguousarray(levels[0]["id"], np.int32).tobytes())
        for ir in range(1, nl + 1):
            for _ in range(npatch[ir]):
                write_record(f, dens)
            for k in FIELDS:
                write_record(f, np.ascontiguousarray(levels[ir][k], np.float32).tobytes())
            write_record(f, np.ascontiguousarray(levels[ir]["id"], np.int32).tobytes())
    if stars is None:
        return
    with open(os.path.join(directory, "clst" + tag), "wb") as f:
        write_record(f, struct.pack("<iff", it, t, zeta))
        write_record(f, dens)
        for k in FIELDS:
            write_record(f, np.ascontiguousarray(sts[0][k], np.float32).tobytes())
        write_record(f, dens)
        write_record(f, dens)
        for ir in range(1, nl + 1):
            for _ in range(npatch[ir]):
                write_record(f, dens)
            s = sts[ir]
            for k in FIELDS:
                write_record(f, np.ascontiguousarray(s[k] if s is not None else [], np.float32).tobytes())
            write_record(f, dens)
            write_record(f, dens)
            write_record(f, np.ascontiguousarray(s["id"] if s is not None else [], np.int32).tobytes())
            z = np.zeros(nbh[ir], np.float32).tobytes()
            for _ in range(7):
                write_record(f, z)
            write_record(f, z)
            write_record(f, np.zeros(nbh[ir], np.int32).tobytes())
