"""The reference's catalogue outputs (asohf.f:800-910): the `familiesNNNNN`
text file and the `particlesNNNNN` unformatted file, plus FRACTION_MASS_SUBS
(substructure.f:1953-1993), which fills their last two columns.

The per-halo rows follow FORMAT 112 of asohf.f:815-818 exactly (Iw, Fw.d and
Ew.d edit descriptors with the Fortran rules: right-justified fields, E
mantissas in [0.1, 1) with a leading "0.", two-digit exponents below 100 and
a field of asterisks when a value does not fit).  The three banner lines
around "NEW ITER" are list-directed in the reference, whose spacing belongs
to the compiler; they are written here in gfortran's layout.  The
`particles` file is a Fortran unformatted sequential file with 4-byte record
markers (gfortran's default): KONTA2; one record (I, first, last) per kept
halo; the largest last index; PARTICLES_PER_HALO up to it.

Positions are written as given: the reference first maps them back to the
input domain (DECONVER_POSITIONS, grids.f:2841), which the caller applies
when its domain differs from the box.
"""
from __future__ import annotations

import re
import struct

import numpy as np

# FORMAT 112, asohf.f:815-818 (51 fields of width 14)
FORMAT_112 = ("2I14,3F14.6,E14.6,F14.6,E14.6,F14.6,2I14,3F14.6,3F14.6,"
              "6E14.6,3E14.6,F14.6,3F14.3,2F14.3,2E14.6,F14.3,E14.3,"
              "F14.6,F14.6,E14.6,F14.6,E14.6,F14.6,E14.6,F14.6,E14.6,"
              "F14.6,E14.6,F14.6,E14.6,F14.6,I14")

HEADER_1 = ["Halo ID", "Substr. of", "Density peak", "coordinates", "(Mpc)", "Virial mass", "Virial radi",
            "Substr. mass", "Substr. radi", "Part. num.", "Most bound", "Center of", "mass coords", "(Mpc)",
            "Semiaxes", "(Mpc)", "", "Inertia", "tensor", "components", "(cMpc^2)", "", "", "Spec. angul.",
            "momentum", "(cMpc km/s)", "Veloc. disp.", "Bulk velocty", "(km/s)", "", "Max part vel",
            "Mean V_rad", "Kinetic E", "Potential E", "Vcmax", "Mass@Vcmax", "r@Vcmax", "R200m (Mpc)",
            "M200m (Msun)", "R200c (Mpc)", "M200c (Msun)", "R500m (Mpc)", "M500m (Msun)", "R500c (Mpc)",
            "M500c (Msun)", "R2500m (Mpc)", "M2500m(Msun)", "R2500c (Mpc)", "M2500c(Msun)", "f_sub", "N_subs"]
HEADER_2 = ["", "", "x", "y", "z", "(Msun)", "(Mpc)", "(Msun)", "(Mpc)", "", "particle ID", "x", "y", "z",
            "Major", "Intermediate", "Minor", "Ixx", "Ixy", "Ixz", "Iyy", "Iyz", "Izz", "Lx", "Ly", "Lz",
            "(km/s)", "Vx", "Vy", "Vz", "(km/s)", "(km/s)", "Msun(km/s)^2", "Msun(km/s)^2", "(km/s)", "(Msun)",
            "(Mpc)"] + [""] * 14
RULE = "=" * 382  # the continued literal of asohf.f:833-839, without fixed-form line padding


def parse_format(fmt: str) -> list[tuple[str, int, int]]:
    """Expands a FORMAT item list ("2I14,3F14.6,E14.6") into (kind, w, d)."""
    out = []
    for item in fmt.split(","):
        m = re.fullmatch(r"(\d*)([IFE])(\d+)(?:\.(\d+))?", item.strip())
        if not m:
            raise ValueError(item)
        rep = int(m.group(1) or 1)
        out += [(m.group(2), int(m.group(3)), int(m.group(4) or 0))] * rep
    return out


def fmt_i(v, w: int) -> str:
    s = str(int(v))
    return s.rjust(w) if len(s) <= w else "*" * w


def fmt_f(v, w: int, d: int) -> str:
    v = float(np.float32(v))
    if not np.isfinite(v):
        s = "NaN" if v != v else ("Infinity" if v > 0 else "-Infinity")
        return s.rjust(w) if len(s) <= w else "*" * w
    s = f"{v:.{d}f}"
    if s.startswith("0.") and len(s) == w + 1:   # the optional leading zero goes first
        s = s[1:]
    elif s.startswith("-0.") and len(s) == w + 1:
        s = "-" + s[2:]
    return s.rjust(w) if len(s) <= w else "*" * w


def fmt_e(v, w: int, d: int) -> str:
    v = float(np.float32(v))
    if not np.isfinite(v):
        s = "NaN" if v != v else ("Infinity" if v > 0 else "-Infinity")
        return s.rjust(w) if len(s) <= w else "*" * w
    sign = "-" if (v < 0 or (v == 0 and np.signbit(v))) else ""
    a = abs(v)
    if a == 0.0:
        digits, exp = "0" * d, 0
    else:
        m, e = f"{a:.{d - 1}e}".split("e")          # d significant digits, correctly rounded
        digits, exp = m.replace(".", ""), int(e) + 1  # 0.ddd form
    es = f"E{'+' if exp >= 0 else '-'}{abs(exp):02d}" if abs(exp) <= 99 else f"{'+' if exp >= 0 else '-'}{abs(exp):03d}"
    s = f"{sign}0.{digits}{es}"
    if len(s) > w:
        s = f"{sign}.{digits}{es}"                   # the optional leading zero goes first
    return s.rjust(w) if len(s) <= w else "*" * w


def format_record(values, fmt: str = FORMAT_112) -> str:
    """One formatted record of `values` under the FORMAT item list `fmt`."""
    eds = parse_format(fmt)
    if len(values) != len(eds):
        raise ValueError(f"{len(values)} values for {len(eds)} edit descriptors")
    out = []
    for v, (k, w, d) in zip(values, eds):
        out.append(fmt_i(v, w) if k == "I" else fmt_f(v, w, d) if k == "F" else fmt_e(v, w, d))
    return "".join(out)


def fraction_mass_subs(cat):
    """FRACTION_MASS_SUBS (substructure.f:1953-1993): FSUB, the mass in
    substructure over the halo's own mass (MASA for haloes, MSUB for
    subhaloes), and NSUBS, the number of direct substructures; REAL*4,
    accumulated in catalogue order."""
    n = cat.nclus
    rc = cat.realclus[:n]
    fsub = np.zeros(n, np.float32)
    nsubs = np.zeros(n, np.int32)
    for i in range(n):
        h = int(rc[i])
        if h > 0:
            fsub[h - 1] = np.float32(fsub[h - 1] + np.float32(cat.msub[i]))
            nsubs[h - 1] += 1
    for i in range(n):
        if rc[i] == -1:
            fsub[i] = np.float32(fsub[i] / np.float32(cat.masa[i]))
        elif rc[i] > 0:
            fsub[i] = np.float32(fsub[i] / np.float32(cat.msub[i]))
    return fsub, nsubs


def halo_row(cat, i: int, uv: float, fsub, nsubs) -> list:
    """The 51 values asohf.f:887-900 writes for halo i (0-based)."""
    f = lambda a: float(np.float32(a))
    uv = np.float32(uv)
    return ([i + 1, int(cat.realclus[i]), f(cat.clusrx[i]), f(cat.clusry[i]), f(cat.clusrz[i]), f(cat.masa[i]),
             f(cat.radio[i]), f(cat.msub[i]), f(cat.rsub[i]), int(cat.dmpclus[i]), int(cat.iplip[i]),
             f(cat.clusrxcm[i]), f(cat.clusrycm[i]), f(cat.clusrzcm[i])]
            + [f(v) for v in np.ravel(cat.eigenval[i])] + [f(v) for v in np.ravel(cat.inertia_tensor[i])]
            + [f(v) for v in np.ravel(cat.angularm[i])]
            + [f(cat.velocity_dispersion[i]), f(cat.vx[i] * uv), f(cat.vy[i] * uv), f(cat.vz[i] * uv),
               f(cat.vmaxclus[i]), f(cat.mean_vr[i]), f(cat.kinetic_e[i]), f(cat.potential_e[i]),
               f(cat.vcmax[i]), f(cat.mcmax[i]), f(cat.rcmax[i]),
               f(cat.r200m[i]), f(cat.m200m[i]), f(cat.r200c[i]), f(cat.m200c[i]),
               f(cat.r500m[i]), f(cat.m500m[i]), f(cat.r500c[i]), f(cat.m500c[i]),
               f(cat.r2500m[i]), f(cat.m2500m[i]), f(cat.r2500c[i]), f(cat.m2500c[i]),
               f(fsub[i]), int(nsubs[i])])


def _list_directed(values) -> str:
    """gfortran's list-directed layout: integers in 12 columns, REAL*4 as
    1PG15.8 style fields, one leading blank."""
    parts = []
    for v in values:
        if isinstance(v, (int, np.integer)):
            parts.append(f"{int(v):12d}")
        else:
            parts.append(f"{float(np.float32(v)):17.8E}" if v != 0 and (abs(v) >= 1e8 or abs(v) < 0.1)
                         else f"{float(np.float32(v)):15.8f}")
    return "".join(parts)


def write_families(path: str, cat, it: int, zeta: float, uv: float) -> int:
    """Writes the families file of asohf.f:812-884; returns the kept haloes."""
    n = cat.nclus
    keep = np.nonzero(cat.realclus[:n] != 0)[0]
    fsub, nsubs = fraction_mass_subs(cat)
    with open(path, "w") as f:
        f.write(" *********************NEW ITER*******************\n")
        f.write(_list_directed([it, n, len(keep), np.float32(zeta)]) + "\n")
        f.write(" ************************************************\n")
        f.write(RULE + "\n")
        f.write("".join(h.rjust(14)[:14] if len(h) <= 14 else h[:14] for h in HEADER_1) + "\n")
        f.write("".join(h.rjust(14)[:14] for h in HEADER_2) + "\n")
        f.write(RULE + "\n")
        for i in keep:
            f.write(format_record(halo_row(cat, int(i), uv, fsub, nsubs)) + "\n")
    return len(keep)


def _record(f, payload: bytes):
    f.write(struct.pack("<i", len(payload)))
    f.write(payload)
    f.write(struct.pack("<i", len(payload)))


def write_particles(path: str, cat, pph) -> None:
    """The unformatted particles file of asohf.f:819-822, 901-909."""
    n = cat.nclus
    keep = np.nonzero(cat.realclus[:n] != 0)[0]
    last = 0
    with open(path, "wb") as f:
        _record(f, struct.pack("<i", len(keep)))
        for i in keep:
            a, b = (int(v) for v in np.ravel(cat.indcs[i]))
            _record(f, struct.pack("<3i", int(i) + 1, a, b))
            last = max(last, b)
        _record(f, struct.pack("<i", last))
        _record(f, np.ascontiguousarray(np.asarray(pph)[:last], np.int32).tobytes())


def read_particles(path: str) -> dict:
    """Reads a particles file: {"haloes": [(I, first, last)], "ids": int32 array}."""
    recs = []
    with open(path, "rb") as f:
        while True:
            h = f.read(4)
            if not h:
                break
            (ln,) = struct.unpack("<i", h)
            body = f.read(ln)
            (tl,) = struct.unpack("<i", f.read(4))
            if tl != ln or len(body) != ln:
                raise ValueError("broken record marker")
            recs.append(body)
    (nkeep,) = struct.unpack("<i", recs[0])
    haloes = [struct.unpack("<3i", r) for r in recs[1:1 + nkeep]]
    (last,) = struct.unpack("<i", recs[1 + nkeep])
    ids = np.frombuffer(recs[2 + nkeep], np.int32).copy()
    if ids.shape[0] != last:
        raise ValueError("ID record length differs from its count")
    return {"haloes": haloes, "ids": ids}


def read_families(path: str) -> np.ndarray:
    """The halo rows of a families file as a (rows, 51) float64 array (the
    fixed 14-column fields of FORMAT 112)."""
    rows = []
    with open(path) as f:
        lines = f.read().splitlines()
    for ln in lines[7:]:
        if not ln.strip():
            continue
        fields = [ln[14 * k:14 * k + 14] for k in range(51)]
        rows.append([float(x.replace("E", "e")) if x.strip() and "*" not in x else np.nan for x in fields])
    return np.array(rows, np.float64).reshape(-1, 51)


def write_outputs(out_dir: str, it: int, cat, pph, zeta: float, uv: float, flag_wdm: int = 1) -> list[str]:
    """The files asohf.f:812-910 writes at the end of iteration `it`:
    output_files/familiesNNNNN and, with FLAG_WDM = 1, particlesNNNNN
    (NNNNN: the iteration as I5.5)."""
    import os
    os.makedirs(out_dir, exist_ok=True)
    tag = f"{it:05d}"
    paths = [os.path.join(out_dir, "families" + tag)]
    write_families(paths[0], cat, it, zeta, uv)
    if flag_wdm == 1:
        paths.append(os.path.join(out_dir, "particles" + tag))
        write_particles(paths[1], cat, pph)
    return paths
