"""Data misfit and its gradient with respect to ln(sigma) of the earth cells,
for Full_Impedance data, on the GPU through the C ABI.

This is the data term of the inversion's penalty functional and its
gradient (func and gradient, f90/INV/INVcore.f90:65-206), with the model
covariance and the regularisation left to the caller (they stay in the
reference's Fortran):

    Phi(m)  = SS / Ndata,   SS = sum |(d - dHat(m)) / err|^2
    grad    = -2 / Ndata * sum_tx J_tx^T ((d - dHat) / err^2)

where dHat are the predicted impedances (fwdPred: one forward solve per
frequency and polarisation, dataResp), Ndata counts real data values (8 per
site and frequency: real and imaginary parts of the four components) and
J_tx^T is JmultT_TX (mt3d_jmult_t: LmultT, the transposed solves, PmultT).
The boundary data of the forward solves are the caller's and are held
fixed, as in the reference's sensitivity, which does not differentiate them.
"""
from __future__ import annotations

import numpy as np


def predict(s, freqs, bcs, sites, origin=(0.0, 0.0, 0.0)):
    """Forward fields and impedances at the handle's model.

    s: capi.Solver with the model set (mt3d_update_cond); freqs [nf] in Hz;
    bcs [nf, 2, nE] boundary data of polarisations 1 and 2; sites [nsite, 3].
    Returns (Z [nf, nsite, 2, 2], E [nf, 2, nE])."""
    freqs = np.asarray(freqs, np.float64)
    nf = freqs.size
    om = np.repeat(2 * np.pi * freqs, 2)
    bc = np.ascontiguousarray(np.asarray(bcs, np.complex128).reshape(2 * nf, -1))
    e, st, rc = s.fwdsolve_batch(om, bc=bc, e0=bc)
    if np.any(st > 1):
        raise RuntimeError(f"forward solves failed: status {st.tolist()}")
    E = e.reshape(nf, 2, -1)
    Z = np.stack([s.impedance(2 * np.pi * f, sites, E[k, 0], E[k, 1], origin=origin) for k, f in enumerate(freqs)])
    return Z, E


def misfit(Z, d_obs, err):
    """(Phi, residual weights (d - dHat) / err^2, Ndata) of Full_Impedance data."""
    res = np.asarray(d_obs) - np.asarray(Z)
    r = res / np.asarray(err)
    ndata = 2 * r.size
    return float(np.sum(np.abs(r) ** 2)) / ndata, res / np.asarray(err) ** 2, ndata


def misfit_gradient(s, m_earth, freqs, bcs, sites, d_obs, err, origin=(0.0, 0.0, 0.0)):
    """Phi and its gradient with respect to ln(sigma) of the earth cells at
    the handle's current model m_earth (already set with update_cond)."""
    Z, E = predict(s, freqs, bcs, sites, origin)
    phi, w, ndata = misfit(Z, d_obs, err)
    grad = np.zeros(np.asarray(m_earth).size)
    for k, f in enumerate(np.asarray(freqs, np.float64)):
        dm, rc = s.jmult_t(2 * np.pi * f, sites, E[k, 0], E[k, 1], w[k], m_earth, origin=origin)
        if rc != 0:
            raise RuntimeError(f"transposed solves at {f} Hz did not converge")
        grad += dm
    return phi, -2.0 / ndata * grad


def taylor_test(s, m_earth, air_cond, dm, freqs, bcs, sites, d_obs, err, origin=(0.0, 0.0, 0.0)):
    """The total-derivative test of the reference's TEST_GRAD job
    (f90/Mod3DMT.f90:297-333) for the data term: f(m0 + dm) - f(m0) against
    grad f(m0) . dm.  Leaves the handle at m0.  Returns (f(m0), the
    difference, the linear prediction)."""
    m0 = np.asarray(m_earth, np.float64)
    s.update_cond(m0, air_cond)
    f1, grad = misfit_gradient(s, m0, freqs, bcs, sites, d_obs, err, origin)
    s.update_cond(m0 + dm, air_cond)
    Z, _ = predict(s, freqs, bcs, sites, origin)
    f2 = misfit(Z, d_obs, err)[0]
    s.update_cond(m0, air_cond)
    return f1, f2 - f1, float(np.dot(grad, dm))


def central_differences(s, m_earth, air_cond, cells, freqs, bcs, sites, d_obs, err, h=1e-4,
                        origin=(0.0, 0.0, 0.0)):
    """(f(m + h e_c) - f(m - h e_c)) / 2h for each earth cell c (flat index
    into m_earth).  Leaves the handle at m."""
    m0 = np.asarray(m_earth, np.float64)
    out = np.zeros(len(cells))
    for n, c in enumerate(cells):
        f = []
        for sign in (1.0, -1.0):
            m = m0.copy()
            m[c] += sign * h
            s.update_cond(m, air_cond)
            Z, _ = predict(s, freqs, bcs, sites, origin)
            f.append(misfit(Z, d_obs, err)[0])
        out[n] = (f[0] - f[1]) / (2 * h)
    s.update_cond(m0, air_cond)
    return out
