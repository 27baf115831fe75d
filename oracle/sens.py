"""The misfit gradient composed from the CPU oracle -- TEST INFRASTRUCTURE ONLY
(the checker of mt3d_jmult_t and mt3d/sens.py).

Restates, with the oracle's forward solver (oracle.py), its transposed solve
and PmultT, and the impedance functional of datafunc.py:
  * fwdPred: one forward solve per frequency and polarisation, dataResp;
  * JmultT_TX (f90/SENS/SensComp.f90:408-488): LmultT -> sensSolve(TRN) ->
    PmultT (f90/3D_MT/SolverSens.f90:63-116), QmultT zero for impedances;
  * the data term of func / gradient (f90/INV/INVcore.f90:65-206):
    Phi = SS / Ndata, grad = -2 / Ndata * sum_tx J^T ((d - dHat) / err^2).
"""
from __future__ import annotations

import numpy as np

from oracle import datafunc
from oracle.oracle import Oracle


def predict(grid, model, freqs, bcs, sites, control, origin=(0.0, 0.0, 0.0)):
    o = Oracle(grid)
    o.update_cond(model.m_earth, model.air_cond)
    o.set_control(**control)
    c = datafunc.coords(grid.dx, grid.dy, grid.dz, grid.nzAir, origin)
    Z, E = [], []
    for k, f in enumerate(np.asarray(freqs, float)):
        om = 2 * np.pi * f
        o.update_freq(om)
        ek = []
        for p in range(2):
            e, rc = o.fwdsolve(bc=bcs[k][p], e0=bcs[k][p])
            if rc != 0:
                raise RuntimeError(f"oracle forward solve failed at {f} Hz")
            ek.append(e)
        E.append(ek)
        Z.append(datafunc.impedance(c, om, sites, ek[0], ek[1]))
    return np.array(Z), E, o, c


def misfit_gradient(grid, model, freqs, bcs, sites, d_obs, err, control, origin=(0.0, 0.0, 0.0)):
    Z, E, o, c = predict(grid, model, freqs, bcs, sites, control, origin)
    res = np.asarray(d_obs) - Z
    ndata = 2 * res.size
    phi = float(np.sum(np.abs(res / err) ** 2)) / ndata
    w = res / np.asarray(err) ** 2
    grad = np.zeros(model.m_earth.size)
    for k, f in enumerate(np.asarray(freqs, float)):
        om = 2 * np.pi * f
        o.update_freq(om)
        s1, s2 = datafunc.lmult_t(c, om, sites, E[k][0], E[k][1], w[k])
        ea = []
        for s in (s1, s2):
            e, rc = o.fwdsolve(trans=True, src=s)
            if rc != 0:
                raise RuntimeError(f"oracle transposed solve failed at {f} Hz")
            ea.append(e)
        grad += o.pmult_t(np.stack(E[k]), np.stack(ea), model.m_earth)
    return phi, -2.0 / ndata * grad


def misfit(grid, model, freqs, bcs, sites, d_obs, err, control, origin=(0.0, 0.0, 0.0)):
    Z, _, _, _ = predict(grid, model, freqs, bcs, sites, control, origin)
    res = np.asarray(d_obs) - Z
    return float(np.sum(np.abs(res / err) ** 2)) / (2 * res.size)
