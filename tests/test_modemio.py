"""ModEM model, control and impedance-data files (mt3d/modemio.py)."""
import os

import numpy as np
import pytest

from mt3d import modemio

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("ptype", ["LOGE", "LOG10", "LINEAR"])
def test_ws_model_round_trip(tmp_path, ptype):
    rng = np.random.default_rng(1)
    dx, dy, dz = rng.uniform(100, 900, 7), rng.uniform(100, 900, 5), rng.uniform(10, 500, 4)
    m = -np.log(10.0) * rng.uniform(0.5, 3.5, 7 * 5 * 4)
    p = tmp_path / "m.rho"
    modemio.write_ws_model(p, dx, dy, dz, m, origin=(-1200.5, 300.25, 0.0), rotation=12.5, param_type=ptype)
    r = modemio.read_ws_model(p)
    assert r["param_type"] == ptype
    assert np.allclose(r["dx"], dx, atol=5e-4) and np.allclose(r["dz_earth"], dz, atol=5e-4)
    # values are written with 6 significant digits (es13.5)
    assert np.allclose(r["m_earth"], m, rtol=2e-5, atol=2e-5)
    assert np.allclose(r["origin"], (-1200.5, 300.25, 0.0)) and r["rotation"] == 12.5


def test_ws_model_layout_x_reversed(tmp_path):
    """One distinct value per cell: row j of layer k lists x from nx down to 1."""
    nx, ny, nz = 3, 2, 2
    m = -np.log(np.arange(1, nx * ny * nz + 1, dtype=float))  # rho = 1..12, x fastest
    p = tmp_path / "l.rho"
    modemio.write_ws_model(p, np.ones(nx), np.ones(ny), np.ones(nz), m, param_type="LINEAR")
    rows = [l.split() for l in open(p).read().split("\n")[6:] if len(l.split()) == nx]
    assert [float(x) for x in rows[0]] == [3.0, 2.0, 1.0] and [float(x) for x in rows[1]] == [6.0, 5.0, 4.0]


def test_model_without_origin_is_centred(tmp_path):
    p = tmp_path / "c.rho"
    p.write_text("# x\n2 2 1 0 LOGE\n100 300\n50 50\n10\n\n1 1\n1 1\n")
    r = modemio.read_ws_model(p)
    assert tuple(r["origin"]) == (-200.0, -50.0, 0.0) and np.all(r["m_earth"] == -1.0)


def test_fwd_control(tmp_path):
    p = tmp_path / "c.fwd"
    lab = lambda s: s.ljust(46) + ": "
    p.write_text("\n".join([lab("Number of QMR iters per divergence correction") + "40",
                            lab("Maximum number of divergence correction calls") + "20",
                            lab("Maximum number of divergence correction iters") + "100",
                            lab("Misfit tolerance for EM forward solver") + "1.0e-7",
                            lab("Misfit tolerance for EM adjoint solver") + "1.0e-7",
                            lab("Misfit tolerance for divergence correction") + "1.0e-5",
                            lab("Optional EM solution file name for nested BC") + "nested.esoln",
                            lab("Air layers mirror|fixed height|read from file") + "fixed height",
                            lab("Number of air layers and min top dz in km") + "12 1000.",
                            lab("Forward solver method PCG|QMR|TFQMR|BICG") + "QMR"]) + "\n")
    c = modemio.read_fwd_control(p)
    assert (c["IterPerDivCor"], c["MaxDivCor"], c["MaxIterDivCor"]) == (40, 20, 100)
    assert c["tolEMfwd"] == 1e-7 and c["tolDivCor"] == 1e-5
    assert c["air_layers"] == dict(method="fixed height", nz=12, params=[1000.0]) and c["solver"] == "QMR"


def test_impedance_units_and_sign():
    """ImpUnits factors and the conjugation of a file with the other sign."""
    assert modemio.imp_units("[V/m]/[T]", "[mV/km]/[nT]") == 1e-3
    assert np.isclose(modemio.imp_units("[mV/km]/[nT]", "Ohm"), 4 * modemio.PI_REF / 10000.0)
    z = np.array([1.0 + 2.0j, -3.0 + 0.5j])
    f = modemio.impedance_to_file(z, "[mV/km]/[nT]", +1)
    assert np.allclose(f, np.conj(z) * 1e-3)
    assert np.allclose(modemio.impedance_from_file(f, "[mV/km]/[nT]", +1), z)
    assert np.allclose(modemio.impedance_from_file(z, "[V/m]/[T]", -1), z)


def test_impedance_data_round_trip_of_the_fixture(tmp_path):
    """The cylinder fixture written in the list format and read back."""
    g = np.load(os.path.join(HERE, "golden", "cylinder_1per.npz"))
    codes = [f"{i // 61 + 1:03d}-{i % 61 + 1:03d}" for i in range(len(g["sites"]))]
    p = tmp_path / "z.dat"
    Z = g["Z"][None]
    Z[0, 5, 1, 1] = np.nan  # an absent component is left out of the file
    modemio.write_impedance_data(p, [float(g["period"])], codes, g["sites"], Z, units="[mV/km]/[nT]", sign=+1,
                                 origin_latlon=(45.0, -90.0))
    d = modemio.read_impedance_data(p)
    assert d["codes"] == codes and d["units"] == "[mV/km]/[nT]" and d["sign"] == +1
    assert np.allclose(d["sites"], g["sites"]) and d["origin_latlon"] == (45.0, -90.0)
    ok = ~np.isnan(Z.real)
    assert np.all(np.isnan(d["Z"].real) == ~ok)
    assert np.allclose(d["Z"][ok], Z[ok], rtol=1e-6, atol=0)
