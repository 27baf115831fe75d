"""Synthetic grids, conductivity models and frequency lists for the 3D-MT solve.

These build the inputs a ModEM run would read from its model and data files:
the staggered grid (cell widths dx, dy, dz with nzAir air layers on top, the
layout of ``grid_t`` in f90/3D_MT/GridDef.f90:18-60) and the model parameter
ln(sigma) of the earth cells (``modelParam_t`` with paramType LOGE,
f90/3D_MT/modelParam/ModelSpace.f90).  Arrays are Fortran ordered (x fastest)
and flattened, matching the reference's column-major storage.

All generators are seeded and deterministic.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

#: f90/UTILS/math_constants.f90:12-19 (PI with the reference's typo; SIGMA_AIR
#: is a single-precision literal promoted to double).
PI_REF = 3.14159265357898
MU_0 = PI_REF * 0.0000004
SIGMA_AIR = float(np.float32(1.0e-10))
#: default air conductivity parameter for LOGE models (ModelSpace.f90:204)
AIR_COND_LOGE = math.log(SIGMA_AIR)


@dataclasses.dataclass
class Grid:
    """Tensor-product staggered grid (f90/3D_MT/GridDef.f90 grid_t)."""

    dx: np.ndarray
    dy: np.ndarray
    dz: np.ndarray  # air layers first (top down), then earth layers
    nzAir: int

    @property
    def nx(self) -> int:
        return int(self.dx.size)

    @property
    def ny(self) -> int:
        return int(self.dy.size)

    @property
    def nz(self) -> int:
        return int(self.dz.size)

    @property
    def nzEarth(self) -> int:
        return self.nz - self.nzAir

    @property
    def n_edges(self) -> int:
        nx, ny, nz = self.nx, self.ny, self.nz
        return nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz

    @property
    def n_interior_edges(self) -> int:
        nx, ny, nz = self.nx, self.ny, self.nz
        return nx * (ny - 1) * (nz - 1) + (nx - 1) * ny * (nz - 1) + (nx - 1) * (ny - 1) * nz

    @property
    def n_nodes(self) -> int:
        return (self.nx + 1) * (self.ny + 1) * (self.nz + 1)

    @property
    def edge_blocks(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        return ((nx, ny + 1, nz + 1), (nx + 1, ny, nz + 1), (nx + 1, ny + 1, nz))


def padded_axis(n_core: int, core_width: float, n_pad: int, growth: float) -> np.ndarray:
    """Uniform core cells with geometrically growing padding on both sides."""
    pad = core_width * growth ** np.arange(1, n_pad + 1)
    return np.concatenate([pad[::-1], np.full(n_core, core_width), pad]).astype(np.float64)


def layered_axis(n: int, first: float, growth: float) -> np.ndarray:
    return (first * growth ** np.arange(n)).astype(np.float64)


def make_grid(nx: int, ny: int, n_air: int, n_earth: int, core: float = 500.0, n_pad: int = 4,
              pad_growth: float = 1.5, air_first: float = 50.0, air_growth: float = 1.5,
              earth_first: float = 50.0, earth_growth: float = 1.2) -> Grid:
    dx = padded_axis(nx - 2 * n_pad, core, n_pad, pad_growth)
    dy = padded_axis(ny - 2 * n_pad, core, n_pad, pad_growth)
    air = layered_axis(n_air, air_first, air_growth)[::-1]  # thinnest next to the surface
    earth = layered_axis(n_earth, earth_first, earth_growth)
    return Grid(dx, dy, np.concatenate([air, earth]), n_air)


def air_layers(dz_earth: np.ndarray, method: str, nz_air: int, *params: float) -> np.ndarray:
    """Air-layer thicknesses (top down) of setup_airlayers
    (f90/3D_MT/GridDef.f90:406-494) from the forward control line
    (f90/3D_MT/FWD/EMsolve3D.f90:687-718; km on input):
      "mirror" alpha min_top_dz: layer j above the surface (j = 1 next to it)
        is alpha**(j-1) times earth layer j, the top one at least min_top_dz;
      "fixed height" max_height: thicknesses growing log-uniformly from the
        first earth layer to a total of max_height."""
    dz_earth = np.asarray(dz_earth, np.float64)
    dz = np.empty(nz_air)
    if method.startswith("mirror"):
        alpha, min_top = params[0], 1000.0 * params[1]
        for iz in range(nz_air, 0, -1):
            j = nz_air - iz + 1
            dz[iz - 1] = (alpha ** (j - 1)) * dz_earth[j - 1]
        if dz[0] < min_top:
            dz[0] = min_top
    elif method.startswith("fixed height"):
        max_height = 1000.0 * params[0]
        z1 = math.log10(dz_earth[0])
        dlog = (math.log10(max_height) - z1) / nz_air
        zl = z1
        for iz in range(nz_air, 0, -1):
            dz[iz - 1] = 10.0 ** (zl + dlog) - 10.0 ** zl
            zl = zl + dlog
    else:
        raise ValueError(f"unknown air-layer method {method!r}")
    return dz


def gaussian_random_field(shape, corr_len_cells: float, seed: int) -> np.ndarray:
    """Zero-mean, unit-variance stationary Gaussian field with exponential
    covariance exp(-|h|/L) (h in cell units), sampled by circulant embedding on
    a grid twice the size in each direction.  Negative eigenvalues of the
    embedding (if any) are clipped to zero.  Returned in Fortran order
    (shape (nx, ny, nz), x fastest when flattened with order='F')."""
    rng = np.random.default_rng(seed)
    ext = [2 * s for s in shape]
    axes = [np.minimum(np.arange(m), m - np.arange(m)).astype(np.float64) for m in ext]
    hx, hy, hz = np.meshgrid(*axes, indexing="ij")
    cov = np.exp(-np.sqrt(hx ** 2 + hy ** 2 + hz ** 2) / corr_len_cells)
    lam = np.fft.fftn(cov).real
    lam = np.clip(lam, 0.0, None)
    noise = rng.standard_normal(ext) + 1j * rng.standard_normal(ext)
    field = np.fft.ifftn(np.sqrt(lam) * noise) * np.sqrt(np.prod(ext))
    f = field.real[: shape[0], : shape[1], : shape[2]]
    f = (f - f.mean()) / (f.std() + 1e-300)
    return f


def random_log10_rho(grid: Grid, seed: int, mean: float = 2.0, std: float = 0.5, corr_len: float = 5.0,
                     clip=(0.0, 4.0)) -> np.ndarray:
    """log10 resistivity of the earth cells, shape (nx, ny, nzEarth)."""
    f = gaussian_random_field((grid.nx, grid.ny, grid.nzEarth), corr_len, seed)
    return np.clip(mean + std * f, clip[0], clip[1])


def loge_from_log10_rho(log10_rho: np.ndarray) -> np.ndarray:
    """ln(sigma) from log10(rho): sigma = 10**-log10_rho."""
    return -np.log(10.0) * log10_rho


def flat_f(a: np.ndarray) -> np.ndarray:
    return np.asfortranarray(a).ravel(order="F").astype(np.float64)


@dataclasses.dataclass
class Model:
    grid: Grid
    m_earth: np.ndarray  # ln(sigma) of earth cells, flattened x fastest
    air_cond: float = AIR_COND_LOGE

    def sigma_cells(self) -> np.ndarray:
        """Cell conductivity (ModelParamToCell), shape (nx, ny, nz)."""
        g = self.grid
        s = np.empty((g.nx, g.ny, g.nz))
        s[:, :, : g.nzAir] = math.exp(self.air_cond)
        s[:, :, g.nzAir:] = np.exp(self.m_earth.reshape((g.nx, g.ny, g.nzEarth), order="F"))
        return s


def halfspace_model(grid: Grid, rho: float) -> Model:
    m = np.full(grid.nx * grid.ny * grid.nzEarth, math.log(1.0 / rho))
    return Model(grid, m)


def block_model(grid: Grid, rho_bg: float, blocks) -> Model:
    """blocks: iterable of (ix0, iy0, iz0_earth, nbx, nby, nbz, rho)."""
    m = np.full((grid.nx, grid.ny, grid.nzEarth), math.log(1.0 / rho_bg))
    for ix0, iy0, iz0, nbx, nby, nbz, rho in blocks:
        m[ix0:ix0 + nbx, iy0:iy0 + nby, iz0:iz0 + nbz] = math.log(1.0 / rho)
    return Model(grid, flat_f(m))


def log_frequencies(n: int, f_lo: float, f_hi: float) -> np.ndarray:
    if n == 1:
        return np.array([f_lo])
    return np.logspace(math.log10(f_lo), math.log10(f_hi), n)


# --------------------------------------------------------------------------
# The benchmark workloads (synthetic inputs with the shapes the solver is
# quoted on).  Seeds are fixed so every run sees the same inputs.
# --------------------------------------------------------------------------

def config_small_forward() -> tuple[Model, np.ndarray]:
    """24x24x24 grid (8 air + 16 earth), 100 ohm-m halfspace with a 1 ohm-m
    4x4x4 block centred, starting at earth layer 3; 0.1 Hz."""
    g = make_grid(24, 24, 8, 16, core=500.0, n_pad=4, pad_growth=1.5, air_first=50.0, air_growth=1.5,
                  earth_first=50.0, earth_growth=1.2)
    c = g.nx // 2 - 2
    m = block_model(g, 100.0, [(c, c, 2, 4, 4, 4, 1.0)])
    return m, np.array([0.1])


def config_precision(seed: int = 20240601) -> tuple[Model, np.ndarray]:
    """100x100x60 (10 air + 50 earth) seeded random field, 1 Hz."""
    g = make_grid(100, 100, 10, 50)
    lr = random_log10_rho(g, seed)
    return Model(g, flat_f(loge_from_log10_rho(lr))), np.array([1.0])


def config_batch(seed: int = 20240602):
    """Three seeded random-field models on 40x40x40, 64x64x48 and 96x96x56,
    8 frequencies log-spaced 1e-3..1e2 Hz each."""
    shapes = [(40, 40, 8, 32), (64, 64, 10, 38), (96, 96, 10, 46)]
    out = []
    for k, (nx, ny, na, ne) in enumerate(shapes):
        g = make_grid(nx, ny, na, ne, earth_growth=1.15)
        lr = random_log10_rho(g, seed + k)
        out.append((Model(g, flat_f(loge_from_log10_rho(lr))), log_frequencies(8, 1e-3, 1e2)))
    return out


def config_gradient(seed: int = 20240603):
    """80x80x50 true model (random field + 0.3 and 1000 ohm-m blocks), 100
    ohm-m starting halfspace, 6 frequencies 1e-3..1e1 Hz."""
    g = make_grid(80, 80, 10, 40, earth_growth=1.15)
    lr = random_log10_rho(g, seed)
    lr[30:38, 30:38, 4:10] = math.log10(0.3)
    lr[44:52, 40:48, 6:14] = math.log10(1000.0)
    true = Model(g, flat_f(loge_from_log10_rho(lr)))
    start = halfspace_model(g, 100.0)
    return true, start, log_frequencies(6, 1e-3, 1e1)


def config_combined(seed: int = 20240604):
    """200x200x100 (12 air + 88 earth) seeded random field, 16 frequencies
    log-spaced 1e-4..1e2 Hz."""
    g = make_grid(200, 200, 12, 88, earth_growth=1.07, air_growth=1.6)
    lr = random_log10_rho(g, seed)
    return Model(g, flat_f(loge_from_log10_rho(lr))), log_frequencies(16, 1e-4, 1e2)
