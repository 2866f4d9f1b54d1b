"""Particle input in the reference's formats: the generic file
(readers/particle_general.f) and GADGET format-2 snapshots
(readers/gadget_unformatted.f).

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
