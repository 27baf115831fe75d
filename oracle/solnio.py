"""E-field solution files restated with the struct module -- TEST
INFRASTRUCTURE ONLY (the checker of mt3d_write_soln / mt3d_read_soln).

Restates the binary layout of write_solnVectorMTX / read_solnVectorMTX
(f90/3D_MT/ioMod/ioAscii.f90:493-597) with FileWriteInit (:188-215),
FileReadInit (f90/3D_MT/ioMod/ioBinary.f90:61-93), EfileWrite (:350-368)
and EfileRead (:314-347), as gfortran writes unformatted sequential files on
a little-endian host: each record framed by its byte length (int32) before
and after; the header record version (character*20), nTx, nMode, nx, ny, nz,
nzAir (integer*4), ox, oy, oz, rotdeg (real*8); then dx, dy, dz; then per
transmitter j and mode k the record (omega, j, k, Pol_name) and the Ex, Ey,
Ez arrays (complex*16, column-major).  Pol_name is 'Ex', 'Ey' for the two MT
polarisations (create_solnVector, f90/3D_MT/SolnSpace.f90:199-205); version
is blank (write_solnVectorMTX).
"""
from __future__ import annotations

import struct

import numpy as np


def _rec(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def _name(s: str) -> bytes:
    return s.encode().ljust(20, b" ")[:20]


def write(path, grid, omegas, fields, origin=(0.0, 0.0, 0.0), rotdeg=0.0):
    """fields: [nTx, nPol, nE] complex, full edge vectors (getCVector order)."""
    fields = np.asarray(fields, np.complex128)
    ntx, npol, ne = fields.shape
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    nX, nY = nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1)
    out = [_rec(_name("") + struct.pack("<6i", ntx, npol, nx, ny, nz, grid.nzAir) +
                struct.pack("<4d", origin[0], origin[1], origin[2], rotdeg))]
    for d in (grid.dx, grid.dy, grid.dz):
        out.append(_rec(np.asarray(d, "<f8").tobytes()))
    for j in range(ntx):
        for k in range(npol):
            name = ("Ex", "Ey")[k] if npol == 2 else ""
            out.append(_rec(struct.pack("<d2i", omegas[j], j + 1, k + 1) + _name(name)))
            e = fields[j, k].astype("<c16")
            for part in (e[:nX], e[nX:nX + nY], e[nX + nY:]):
                out.append(_rec(part.tobytes()))
    with open(path, "wb") as f:
        f.write(b"".join(out))


def _records(path):
    data = open(path, "rb").read()
    p, recs = 0, []
    while p < len(data):
        (n,) = struct.unpack_from("<i", data, p)
        recs.append(data[p + 4:p + 4 + n])
        (m,) = struct.unpack_from("<i", data, p + 4 + n)
        assert m == n, "record markers differ"
        p += 8 + n
    return recs


def read(path):
    """(header dict, omegas [nTx], fields [nTx, nPol, nE], names [nTx][nPol])."""
    recs = _records(path)
    h = recs[0]
    version = h[:20].decode()
    ntx, npol, nx, ny, nz, nza = struct.unpack_from("<6i", h, 20)
    ox, oy, oz, rot = struct.unpack_from("<4d", h, 44)
    dx, dy, dz = (np.frombuffer(r, "<f8").copy() for r in recs[1:4])
    omegas, fields, names = np.zeros(ntx), [], []
    for j in range(ntx):
        row, nrow = [], []
        for k in range(npol):
            r = recs[4 + (j * npol + k) * 4]
            om, jj, kk = struct.unpack_from("<d2i", r, 0)
            assert (jj, kk) == (j + 1, k + 1)
            omegas[j] = om
            nrow.append(r[16:36].decode().strip())
            row.append(np.concatenate([np.frombuffer(recs[5 + (j * npol + k) * 4 + c], "<c16") for c in range(3)]))
        fields.append(row)
        names.append(nrow)
    head = dict(version=version, nTx=ntx, nPol=npol, nx=nx, ny=ny, nz=nz, nzAir=nza, origin=(ox, oy, oz),
                rotdeg=rot, dx=dx, dy=dy, dz=dz)
    return head, omegas, np.array(fields), names
