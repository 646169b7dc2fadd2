"""Synthetic photonic geometries and excitations (inputs of the VIE solve).

These generate the seeded synthetic workloads of the benchmark configurations:
a straight Si strip, Bragg gratings with quadratic absorbers and a microdisk
with a bus waveguide, all as voxelised relative permittivities (Si relative
to the SiO2 background, as Bragg_params_heat_lengthways.m:21-23 scales by
n_ext).  They follow the construction of Bragg_geometry.m:4-42 and
generatedomain_begin_at_x_eq_0.m:79-97 (voxel centres on a regular grid,
membership tested at the centres); material values follow the benchmark
definitions (eps_Si = 12.11, eps_SiO2 = 2.085, absorber Im(eps_r) ramped
quadratically from 0 to 0.5) rather than the reference's Lorentz model.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

C0 = 299792458.0
MU0 = 4 * np.pi * 1e-7
EPS0 = 1.0 / C0 ** 2 / MU0
EPS_SI = 12.11
EPS_SIO2 = 2.085
N_EXT = float(np.sqrt(EPS_SIO2))


@dataclass
class Problem:
    """A voxelised scatterer in a homogeneous background."""
    name: str
    res: float                 # voxel edge (m)
    e_r: np.ndarray            # L x M x N relative permittivity (complex)
    centres: tuple             # (x, y, z) 1-D coordinate arrays of voxel centres
    lam0: float = 1550e-9      # free-space wavelength
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return self.e_r.shape

    @property
    def Gram(self):
        return self.res ** 3

    @property
    def freq(self):
        # background-medium frequency convention of Si_in_SiO2_parameters.m:18
        return C0 / self.lam0 * N_EXT

    @property
    def ko(self):
        return 2 * np.pi * self.freq / C0

    def idxS(self):
        """1-based column-major positions of non-background voxels."""
        Mc = self.e_r - 1.0
        return np.flatnonzero(np.abs(Mc.reshape(-1, order="F")) > 1e-12) + 1

    def idxS3(self):
        s = self.idxS()
        V = self.e_r.size
        return np.concatenate([s, V + s, 2 * V + s])

    def Mop(self):
        """Mc ./ Mr of the JVIE-II form, (e_r - 1) / e_r."""
        return (self.e_r - 1.0) / self.e_r

    def with_wavelength(self, lam0):
        return Problem(self.name, self.res, self.e_r, self.centres, lam0, dict(self.meta))


def _grid(res, Lx, Wy, Hz):
    nx, ny, nz = (max(1, int(round(v / res))) for v in (Lx, Wy, Hz))
    x = (np.arange(nx) + 0.5) * res
    y = (np.arange(ny) - (ny - 1) / 2.0) * res
    z = (np.arange(nz) - (nz - 1) / 2.0) * res
    return x, y, z


def strip(length=2e-6, width=500e-9, height=220e-9, res=20e-9, lam0=1550e-9):
    """Straight Si strip filling the whole grid (100 x 25 x 11 at 20 nm)."""
    x, y, z = _grid(res, length, width, height)
    e_r = np.full((x.size, y.size, z.size), EPS_SI / EPS_SIO2, dtype=complex)
    return Problem("strip", res, e_r, (x, y, z), lam0)


def bragg(periods=60, period=320e-9, duty=0.5, width=500e-9, corrugation=25e-9,
          height=220e-9, len_abs=2e-6, res=20e-9, M=None, lam0=1550e-9, abs_im=0.5):
    """Bragg grating with quadratic absorbers at both ends.

    Section lengths follow Bragg_geometry.m:4 (2 absorbers + periods); the
    grating alternates wide (width + 2*corrugation ... here width/2 +
    corrugation half-width) and narrow sections over each period; the
    absorbers are straight waveguide whose Im(eps_r) ramps quadratically from
    0 at the inner edge to -abs_im at the domain ends (Bragg_params_heat_lengthways.m:56-73
    shape, benchmark magnitude).
    """
    length = 2 * len_abs + periods * period
    if M is None:
        M = int(round((width + 2 * corrugation) / res)) + 2
    x, _, z = _grid(res, length, M * res, height)
    y = (np.arange(M) - (M - 1) / 2.0) * res
    L, N = x.size, z.size
    X, Y = np.meshgrid(x, y, indexing="ij")
    xs, xe = len_abs, len_abs + periods * period
    half = np.full(X.shape, width / 2)
    in_grating = (X >= xs) & (X < xe)
    phase = np.mod(X - xs, period)
    wide = in_grating & (phase < duty * period)
    narrow = in_grating & ~wide
    half = np.where(wide, width / 2 + corrugation, half)
    half = np.where(narrow, width / 2 - corrugation, half)
    tol = 1e-3 * res
    si2d = np.abs(Y) <= half + tol
    e2d = np.where(si2d, EPS_SI / EPS_SIO2, 1.0).astype(complex)
    ramp = np.zeros_like(X)
    ramp = np.where(X <= len_abs, ((len_abs - X) / len_abs) ** 2, ramp)
    ramp = np.where(X >= length - len_abs, ((X - (length - len_abs)) / len_abs) ** 2, ramp)
    e2d = np.where(si2d, e2d - 1j * abs_im * ramp, e2d)
    e_r = np.repeat(e2d[:, :, None], N, axis=2)
    return Problem("bragg", res, e_r, (x, y, z), lam0,
                   {"periods": periods, "len_abs": len_abs, "width": width,
                    "corrugation": corrugation})


def microdisk(radius=5e-6, gap=200e-9, bus_width=500e-9, height=220e-9, len_abs=2e-6,
              res=20e-9, L=560, M=540, lam0=1550e-9, abs_im=0.5):
    """Si microdisk side-coupled to a bus waveguide (560 x 540 x 11 at 20 nm)."""
    x = (np.arange(L) - (L - 1) / 2.0) * res
    y = (np.arange(M) - (M - 1) / 2.0) * res
    z = (np.arange(int(round(height / res))) - (int(round(height / res)) - 1) / 2.0) * res
    X, Y = np.meshgrid(x, y, indexing="ij")
    ybus = y[0] + bus_width / 2 + res
    disk_c = ybus + bus_width / 2 + gap + radius
    disk = (X ** 2 + (Y - disk_c) ** 2) <= radius ** 2
    bus = np.abs(Y - ybus) <= bus_width / 2
    si = disk | bus
    e2d = np.where(si, EPS_SI / EPS_SIO2, 1.0).astype(complex)
    xl = x[0] - res / 2
    xr = x[-1] + res / 2
    ramp = np.zeros_like(X)
    ramp = np.where(X <= xl + len_abs, ((xl + len_abs - X) / len_abs) ** 2, ramp)
    ramp = np.where(X >= xr - len_abs, ((X - (xr - len_abs)) / len_abs) ** 2, ramp)
    e2d = np.where(bus, e2d - 1j * abs_im * ramp, e2d)
    e_r = np.repeat(e2d[:, :, None], z.size, axis=2)
    return Problem("microdisk", res, e_r, (x, y, z), lam0,
                   {"radius": radius, "gap": gap, "bus_width": bus_width, "ybus": ybus,
                    "disk_c": disk_c, "len_abs": len_abs})


def microdisk_regions(p: Problem):
    """The preconditioner's sub-domains of the resonator (resonator_MOR_scripts.m:
    45-56 bus box, 115-124 disk square, 170-186 disk voxels), as 1-based
    column-major positions in the whole grid (single component; x3 for the
    three components as the reference's idx_*3):

    * bus: every voxel of the rows (y) of the bus waveguide, L x M_WG x N;
    * square: the x range |x - x_disk| <= radius and the rows above the bus and
      the gap, L_D x M_D x N (the level-2 grid);
    * disk: the disk's voxels in the whole grid, and in the square's grid.
    """
    x, y, z = p.centres
    L, M, N = p.shape
    mt = p.meta
    yb = np.flatnonzero(np.abs(y - mt["ybus"]) <= mt["bus_width"] / 2)
    xs = np.flatnonzero(np.abs(x) <= mt["radius"])
    ys = np.flatnonzero(y >= mt["ybus"] + mt["bus_width"] / 2 + mt["gap"])
    X, Y = np.meshgrid(x, y, indexing="ij")
    disk2 = (X ** 2 + (Y - mt["disk_c"]) ** 2) <= mt["radius"] ** 2

    def positions(xi, yi, mask2=None):
        g = np.zeros((L, M, N), dtype=bool)
        sub = np.zeros((L, M), dtype=bool)
        sub[np.ix_(xi, yi)] = True
        if mask2 is not None:
            sub &= mask2
        g[:, :, :] = sub[:, :, None]
        return np.flatnonzero(g.reshape(-1, order="F")) + 1

    idx_bus = positions(np.arange(L), yb)
    idx_square = positions(xs, ys)
    idx_disk = positions(xs, ys, disk2)
    sq_mask = disk2[np.ix_(xs, ys)]
    sq3 = np.repeat(sq_mask[:, :, None], N, axis=2)
    idx_disk_in_sq = np.flatnonzero(sq3.reshape(-1, order="F")) + 1
    return {"bus": (int(yb[0]), int(yb.size)), "idx_bus": idx_bus,
            "square": (int(xs[0]), int(xs.size), int(ys[0]), int(ys.size)),
            "idx_square": idx_square, "idx_disk": idx_disk, "idx_disk_in_sq": idx_disk_in_sq}


def ext3(idx, V):
    """[idx; V + idx; 2V + idx] (the three Cartesian components)."""
    idx = np.asarray(idx)
    return np.concatenate([idx, V + idx, 2 * V + idx])


def plane_wave(p: Problem, k_dir=(1.0, 0.0, 0.0), Eo=(0.0, 1.0, 0.0)):
    """PlaneWave_Excitation.m:67-98: voxel-averaged plane wave, L x M x N x 3.

    k = ko * k_dir (background wavenumber); each axis factor is the average of
    exp(-j k_a a) over the voxel, normalised by the voxel volume.
    """
    x, y, z = p.centres
    k = p.ko * np.asarray(k_dir, dtype=float)
    dx = p.res

    def axis_factor(ka, a):
        if ka != 0:
            return np.exp(-1j * ka * a) * (np.exp(-1j * ka * dx / 2) - np.exp(1j * ka * dx / 2)) \
                / (-1j * ka)
        return dx * np.ones_like(a, dtype=complex)

    fx = axis_factor(k[0], x)[:, None, None]
    fy = axis_factor(k[1], y)[None, :, None]
    fz = axis_factor(k[2], z)[None, None, :]
    Eexc = fx * fy * fz / dx ** 3
    return np.stack([Eo[0] * Eexc, Eo[1] * Eexc, Eo[2] * Eexc], axis=3)


def bragg_config(name):
    """The benchmark grids: cfg1 strip, cfg2 Bragg 20 nm, cfg3 Bragg 10 nm."""
    if name == "strip":
        return strip()
    if name == "bragg20":
        return bragg(res=20e-9, M=30)
    if name == "bragg10":
        return bragg(res=10e-9, M=60)
    if name.startswith("bragg20-p"):  # e.g. bragg20-p20: 20 periods -> 520 x 30 x 11
        return bragg(periods=int(name[len("bragg20-p"):]), res=20e-9, M=30)
    raise KeyError(name)


def sweep_problems(periods=(20, 40, 60, 80, 100), n_lambda=201, lam_range=(1500e-9, 1600e-9)):
    """The mixed-length sweep: every period count at n_lambda wavelengths."""
    lams = np.linspace(lam_range[0], lam_range[1], n_lambda)
    base = {p: bragg(periods=p, M=30) for p in periods}
    return [(p, lam, base[p].with_wavelength(lam)) for p in periods for lam in lams]
