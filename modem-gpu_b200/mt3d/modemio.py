"""ModEM's model, forward-control and impedance-data files, for running the
device chain on a ModEM user's inputs.

  * WS model files: read_modelParam_ws / write_modelParam_ws
    (f90/3D_MT/modelParam/modelParamIO/WS.inc:4-209): header ``nx ny nzEarth 0
    TYPE``, the cell widths, then per layer and per row the values with x
    reversed, then the grid origin (m) and rotation (deg).  LOGE / LOG10
    files hold ln / log10 of the resistivity, LINEAR files the resistivity.
  * Forward control files: readEMsolveControl
    (f90/3D_MT/FWD/EMsolve3D.f90:580-760): one value per line after a
    48-character label, including the air-layer method.
  * Full_Impedance data files in list format (read / write_dataVectorMTX,
    f90/3D_MT/DataIO.f90:230-900): ``>`` header lines with the data type,
    sign convention, units, orientation, geographic origin and the counts,
    then one line per period, site and component.
  * ImpUnits (f90/3D_MT/DICT/dataTypes.f90:252-315) and the sign handling of
    DataIO (:276-280): impedance_from_file / impedance_to_file convert between
    a file's values and the library's SI E/B impedances with ISIGN = -1
    (the convention of mt3d_impedance).

Arrays of model values are flattened x fastest, like the library's model
parameter (ln sigma of the earth cells).
"""
from __future__ import annotations

import math

import numpy as np

#: f90/UTILS/math_constants.f90:12 (the reference's PI)
PI_REF = 3.14159265357898
ISIGN = -1
_COMPONENTS = ("ZXX", "ZXY", "ZYX", "ZYY")


# --------------------------------------------------------------------------
# model files
# --------------------------------------------------------------------------
def read_ws_model(path) -> dict:
    """dict(dx, dy, dz_earth, m_earth (ln sigma, x fastest), origin, rotation,
    param_type).  Without an origin line the grid is centred as the reference
    does (-sum(dx)/2, -sum(dy)/2, 0)."""
    with open(path) as f:
        lines = f.read().split("\n")
    head = lines[1].split()
    nx, ny, nz = int(head[0]), int(head[1]), int(head[2])
    if int(head[3]) != 0:
        raise ValueError("mapping not supported (as in read_modelParam_ws)")
    up = lines[1].upper()
    ptype = "LOGE" if "LOGE" in up else "LOG10" if "LOG10" in up else "LINEAR"
    toks = " ".join(lines[2:]).split()
    p = 0
    dx = np.array(toks[p:p + nx], float); p += nx
    dy = np.array(toks[p:p + ny], float); p += ny
    dz = np.array(toks[p:p + nz], float); p += nz
    v = np.array(toks[p:p + nx * ny * nz], float).reshape(nz, ny, nx)[:, :, ::-1]
    p += nx * ny * nz
    if len(toks) >= p + 3:
        origin = np.array(toks[p:p + 3], float); p += 3
    else:
        origin = np.array([-dx.sum() / 2.0, -dy.sum() / 2.0, 0.0])
    rot = float(toks[p]) if len(toks) > p else 0.0
    rho = np.transpose(v, (2, 1, 0))  # [nx, ny, nz]
    if ptype == "LOGE":
        m = -rho
    elif ptype == "LOG10":
        m = -rho * math.log(10.0)
    else:
        m = -np.log(rho)
    return dict(dx=dx, dy=dy, dz_earth=dz, m_earth=m.ravel(order="F"), origin=origin, rotation=rot,
                param_type=ptype)


def write_ws_model(path, dx, dy, dz_earth, m_earth, origin=(0.0, 0.0, 0.0), rotation=0.0, param_type="LOGE",
                   comment="3D MT model written by ModEM in WS format"):
    """Writes ln sigma (x fastest) as write_modelParam_ws does."""
    dx, dy, dz = (np.asarray(a, float) for a in (dx, dy, dz_earth))
    nx, ny, nz = dx.size, dy.size, dz.size
    m = np.asarray(m_earth, float).reshape(nx, ny, nz, order="F")
    if param_type == "LOGE":
        v = -m
    elif param_type == "LOG10":
        v = -m / math.log(10.0)
    elif param_type == "LINEAR":
        v = np.exp(-m)
    else:
        raise ValueError(f"unknown parameter type {param_type!r}")
    out = [f" # {comment}", f"{nx:5d}{ny:5d}{nz:5d}{0:5d} {param_type}"]
    for d in (dx, dy, dz):
        out.append("".join(f"{x:12.3f}" for x in d))
    out.append("")
    for k in range(nz):
        for j in range(ny):
            out.append("".join(f"{v[i, j, k]:13.5E}" for i in range(nx - 1, -1, -1)))
        out.append("")
    out.append("".join(f"{x:16.3f}" for x in origin))
    out.append(f"{rotation:9.3f}")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


# --------------------------------------------------------------------------
# forward control files
# --------------------------------------------------------------------------
def read_fwd_control(path) -> dict:
    """The values of a forward control file: IterPerDivCor, MaxDivCor,
    MaxIterDivCor, tolEMfwd, tolEMadj, tolDivCor, the nested-BC file name,
    the air-layer method with its numbers, and the solver name."""
    vals = []
    with open(path) as f:
        for line in f:
            if line.strip():
                vals.append(line[48:].strip() if len(line) > 48 and ":" in line[:49] else line.split(":", 1)[-1].strip())
    out = dict(IterPerDivCor=int(vals[0]), MaxDivCor=int(vals[1]), MaxIterDivCor=int(vals[2]),
               tolEMfwd=float(vals[3]), tolEMadj=float(vals[4]), tolDivCor=float(vals[5]))
    rest = vals[6:]
    if rest:
        out["nested_bc_file"] = rest[0]
    if len(rest) > 2:
        method = rest[1]
        nums = [float(x) for x in rest[2].split()]
        out["air_layers"] = dict(method=method, nz=int(nums[0]), params=nums[1:])
    if len(rest) > 3:
        out["solver"] = rest[3].split()[0]
    return out


# --------------------------------------------------------------------------
# impedance data files
# --------------------------------------------------------------------------
def imp_units(old: str, new: str) -> float:
    """ImpUnits: the factor that takes impedances in `old` units to `new`."""
    def to_si(u):  # [V/m]/[T] per unit of u
        if "[V/m]/[T]" in u:
            return 1.0
        if "[mV/km]/[nT]" in u:
            return 1000.0
        if "[V/m]/[A/m]" in u or "Ohm" in u:
            return 1000.0 * 10000.0 / (4 * PI_REF)
        raise ValueError(f"unknown impedance units {u!r}")
    return to_si(old) / to_si(new)


def impedance_from_file(Z, units: str, sign: int) -> np.ndarray:
    """File values -> SI E/B with ISIGN = -1 (the library's convention)."""
    Z = np.asarray(Z, complex) * imp_units(units, "[V/m]/[T]")
    return Z if sign == ISIGN else np.conj(Z)


def impedance_to_file(Z, units: str = "[mV/km]/[nT]", sign: int = +1) -> np.ndarray:
    """SI E/B with ISIGN = -1 -> values for a file in `units` with `sign`."""
    Z = np.asarray(Z, complex) * imp_units("[V/m]/[T]", units)
    return Z if sign == ISIGN else np.conj(Z)


def read_impedance_data(path) -> dict:
    """dict(periods [np], codes [ns], latlon [ns, 2], sites [ns, 3],
    Z [np, ns, 2, 2], err [np, ns, 2, 2] (NaN where a component is absent),
    units, sign, orientation, origin_latlon, comments)."""
    header, recs = [], []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or line.startswith(">") or line.startswith("+"):
                header.append(line.rstrip("\n"))
                continue
            t = line.split()
            if len(t) >= 11:
                recs.append(t)
    hdr = [h[1:].strip() for h in header if h.startswith(">")]
    if not hdr or "Full_Impedance" not in hdr[0]:
        raise ValueError("not a Full_Impedance data block")
    sign = +1 if "+" in hdr[1] else -1
    units = hdr[2]
    orientation = float(hdr[3].split()[0])
    origin_latlon = tuple(float(x) for x in hdr[4].split()[:2])
    periods = sorted({float(t[0]) for t in recs})
    codes, site_of = [], {}
    for t in recs:
        if t[1] not in site_of:
            site_of[t[1]] = len(codes)
            codes.append((t[1], float(t[2]), float(t[3]), float(t[4]), float(t[5]), float(t[6])))
    Z = np.full((len(periods), len(codes), 2, 2), np.nan + 0j)
    E = np.full((len(periods), len(codes), 2, 2), np.nan)
    pidx = {p: i for i, p in enumerate(periods)}
    for t in recs:
        c = _COMPONENTS.index(t[7].upper())
        i, s = pidx[float(t[0])], site_of[t[1]]
        Z[i, s, c // 2, c % 2] = complex(float(t[8]), float(t[9]))
        E[i, s, c // 2, c % 2] = float(t[10])
    return dict(periods=np.array(periods), codes=[c[0] for c in codes],
                latlon=np.array([c[1:3] for c in codes]), sites=np.array([c[3:6] for c in codes]),
                Z=Z, err=E, units=units, sign=sign, orientation=orientation, origin_latlon=origin_latlon,
                comments=[h for h in header if h.startswith("#")])


def write_impedance_data(path, periods, codes, sites, Z, err=None, latlon=None, units="[mV/km]/[nT]", sign=+1,
                         orientation=0.0, origin_latlon=(0.0, 0.0), comment="ModEM impedance responses"):
    """Z [np, ns, 2, 2] in file units and sign (see impedance_to_file)."""
    Z = np.asarray(Z, complex)
    npd, ns = Z.shape[:2]
    err = np.full(Z.shape, 1.0e13) if err is None else np.asarray(err, float)
    latlon = np.zeros((ns, 2)) if latlon is None else np.asarray(latlon, float)
    out = [f"# {comment}", "# Period(s) Code GG_Lat GG_Lon X(m) Y(m) Z(m) Component Real Imag Error",
           "> Full_Impedance", "> exp(+i\\omega t)" if sign > 0 else "> exp(-i\\omega t)", f"> {units}",
           f"> {orientation:8.2f}", f"> {origin_latlon[0]:9.3f}{origin_latlon[1]:9.3f}", f"> {npd:6d}{ns:6d}"]
    for s in range(ns):  # by receiver, then transmitter, as write_dataVectorMTX orders them
        for i in range(npd):
            for c, name in enumerate(_COMPONENTS):
                z = Z[i, s, c // 2, c % 2]
                if np.isnan(z.real):
                    continue
                out.append(f"{periods[i]:13.6E} {codes[s]:>20s} {latlon[s, 0]:8.3f} {latlon[s, 1]:8.3f} "
                           f"{sites[s][0]:15.3f}{sites[s][1]:15.3f}{sites[s][2]:15.3f} {name:>6s} "
                           f"{z.real:14.6E} {z.imag:14.6E} {err[i, s, c // 2, c % 2]:14.6E}")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
