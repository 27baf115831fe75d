"""Generate tests/golden/cylinder_1per.npz from the reference's unit-test files.

Reads, from the ModEM-GPU source tree (default /root/reference, or the path in
the first argument):
  * unit_testing/3D/CylinderModel+QuarterSpace.rho -- the model (WS format,
    read as read_modelParam_ws does, f90/3D_MT/modelParam/modelParamIO/
    WS.inc:4-121: each row of a layer is stored with x reversed, LOGE values
    are ln(rho), so ln(sigma) = -value; the grid origin follows the values);
  * unit_testing/3D/CylinderModel_1per.dat -- Full_Impedance at 2501 sites
    for one period, written by the reference's forward run
    (unit_testing/3D/unit_testing_level0.sh:40) in [mV/km]/[nT] with the
    exp(+i omega t) sign convention;
  * unit_testing/3D/CylinderModel.fwd -- the air-layer control line.
Writes the grid, ln(sigma) of the earth cells in x-fastest order, the site
coordinates and the impedances exactly as the file gives them.
"""
from __future__ import annotations

import os
import sys

import numpy as np


def read_ws(path):
    with open(path) as f:
        lines = f.read().split("\n")
    head = lines[1].split()
    nx, ny, nz = int(head[0]), int(head[1]), int(head[2])
    assert "LOGE" in lines[1]
    toks = " ".join(lines[2:]).split()
    p = 0
    dx = np.array(toks[p:p + nx], float); p += nx
    dy = np.array(toks[p:p + ny], float); p += ny
    dz = np.array(toks[p:p + nz], float); p += nz
    v = np.array(toks[p:p + nx * ny * nz], float).reshape(nz, ny, nx)[:, :, ::-1]  # x reversed per row
    p += nx * ny * nz
    origin = np.array(toks[p:p + 3], float); p += 3
    rot = float(toks[p]) if p < len(toks) else 0.0
    m = -np.transpose(v, (2, 1, 0))  # [nx, ny, nz], ln(sigma) = -ln(rho)
    return dx, dy, dz, m, origin, rot


def read_dat(path):
    period, sites, z = None, [], {}
    header = []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or line.startswith(">") or line.startswith("+"):
                header.append(line.rstrip())
                continue
            t = line.split()
            if len(t) < 11:
                continue
            per, code = float(t[0]), t[1]
            x, y, zz = float(t[4]), float(t[5]), float(t[6])
            comp, re, im = t[7], float(t[8]), float(t[9])
            period = per if period is None else period
            assert per == period
            if code not in z:
                z[code] = {}
                sites.append((code, x, y, zz))
            z[code][comp] = complex(re, im)
    xyz = np.array([s[1:] for s in sites])
    Z = np.array([[[z[s[0]]["ZXX"], z[s[0]]["ZXY"]], [z[s[0]]["ZYX"], z[s[0]]["ZYY"]]] for s in sites])
    return period, xyz, Z, header


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    d = os.path.join(ref, "unit_testing", "3D")
    dx, dy, dz, m, origin, rot = read_ws(os.path.join(d, "CylinderModel+QuarterSpace.rho"))
    period, xyz, Z, header = read_dat(os.path.join(d, "CylinderModel_1per.dat"))
    assert any("[mV/km]/[nT]" in h for h in header) and any("exp(+i\\omega t)" in h for h in header)
    with open(os.path.join(d, "CylinderModel.fwd")) as f:
        air = [l for l in f if l.startswith("Air layers") or l.startswith("Number of air layers")]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cylinder_1per.npz")
    np.savez_compressed(out, dx=dx, dy=dy, dz_earth=dz, m_earth=m.ravel(order="F"), origin=origin,
                        rotation=rot, period=period, sites=xyz, Z=Z, units="[mV/km]/[nT]", sign=+1,
                        air_control=np.array([a.split(":", 1)[1].strip() for a in air]))
    print(out, os.path.getsize(out), "bytes;", len(xyz), "sites; grid", m.shape)


if __name__ == "__main__":
    main()
