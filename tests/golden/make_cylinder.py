"""Generate tests/golden/cylinder_1per.npz from the reference's unit-test files.

Reads, with the readers of mt3d/modemio.py, from the ModEM-GPU source tree
(default /root/reference, or the path in the first argument):
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

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..", "modem-gpu_b200"))
from mt3d import modemio  # noqa: E402


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
    d = os.path.join(ref, "unit_testing", "3D")
    mod = modemio.read_ws_model(os.path.join(d, "CylinderModel+QuarterSpace.rho"))
    assert mod["param_type"] == "LOGE"
    dat = modemio.read_impedance_data(os.path.join(d, "CylinderModel_1per.dat"))
    assert dat["units"] == "[mV/km]/[nT]" and dat["sign"] == +1 and dat["periods"].size == 1
    period, xyz, Z = float(dat["periods"][0]), dat["sites"], dat["Z"][0]
    with open(os.path.join(d, "CylinderModel.fwd")) as f:
        air = [l for l in f if l.startswith("Air layers") or l.startswith("Number of air layers")]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cylinder_1per.npz")
    np.savez_compressed(out, dx=mod["dx"], dy=mod["dy"], dz_earth=mod["dz_earth"], m_earth=mod["m_earth"],
                        origin=mod["origin"], rotation=mod["rotation"], period=period, sites=xyz, Z=Z,
                        units=dat["units"], sign=dat["sign"],
                        air_control=np.array([a.split(":", 1)[1].strip() for a in air]))
    print(out, os.path.getsize(out), "bytes;", len(xyz), "sites; grid", (mod["dx"].size, mod["dy"].size,
                                                                           mod["dz_earth"].size))


if __name__ == "__main__":
    main()
