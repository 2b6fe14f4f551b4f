"""Synthetic ROMS-shaped grids, hydrodynamic frames and particle releases.

The reference reads its grid (grid_module.f90:41-499) and its hourly frames
(hydrodynamic_module.f90:112-760, ``updateHydro``) from ROMS NetCDF output.
No ocean-model output exists on this machine, so the workloads are analytic
fields with the shapes, sizes and value ranges of the published benchmark
configurations:

* s-coordinates: ROMS ``Vtransform=2`` / ``Vstretching=4`` stretching
  (published ROMS formulas; the reference reads ``Cs_r``/``Cs_w`` from the
  file, grid_module.f90:350-373, and never computes them itself);
* bathymetry ``h = 20 + 180 (1 - exp(-x / 30 km))``;
* velocity: a time-dependent double gyre plus a progressive M2 tide, peak
  speed ~0.3 m/s; ``w`` from continuity of the divergent (tidal) part;
* ``zeta``: M2 wave of 0.5 m amplitude;
* ``AKs``: parabolic in depth, peak 1e-2 m^2/s, tidally modulated;
* optional Stokes drift ``0.05 m/s * exp(z / 5 m)``.

Every array is returned in Fortran (column-major) order with the reference's
shapes: ``h(xi_rho, eta_rho)``, ``u(xi_u, eta_u, N)``, ``v(xi_v, eta_v, N)``,
``w/AKs(xi_rho, eta_rho, N+1)``, ``zeta(xi_rho, eta_rho)``.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Optional

import numpy as np

M2_PERIOD = 44712.0  # s


@dataclasses.dataclass
class GridSpec:
    xi_rho: int
    eta_rho: int
    N: int
    vtransform: int = 2
    theta_s: float = 5.0
    theta_b: float = 0.4
    hc: float = 10.0
    dx: float = 1000.0
    dy: float = 1000.0
    land: str = "corner"          # "corner" | "islands" | "none"
    land_frac: float = 0.08
    land_seed: int = 0
    stokes: bool = False
    eddy: float = 0.0             # extra submesoscale eddy amplitude (m/s)
    field_dtype: str = "f64"      # storage precision of frames: f64 | f32
    x0: float = 0.0               # physical offset of rho point (1,1) (m)
    y0: float = 0.0
    gyre_lx: Optional[float] = None   # gyre domain size; default: this grid
    gyre_ly: Optional[float] = None
    diag: bool = False            # frames also carry salt, temp, bustr, bvstr
    wetdry: bool = False          # frames also carry wet/dry masks (an intertidal flat)
    behave: bool = False          # frames also carry behave's acceleration / vorticity fields

    @property
    def xi_u(self) -> int:
        return self.xi_rho - 1

    @property
    def eta_v(self) -> int:
        return self.eta_rho - 1


def s_coordinate(N: int, theta_s: float, theta_b: float):
    """ROMS Vstretching=4 s-coordinate and stretching curves.

    Returns ``(s_rho[N], Cs_r[N], s_w[N+1], Cs_w[N+1])`` ordered bottom to
    top, the order the reference's ``getSlevel``/``getWlevel`` index them
    (grid_module.f90:513-598).
    """
    def stretch(s):
        if theta_s > 0:
            c = (1.0 - np.cosh(theta_s * s)) / (np.cosh(theta_s) - 1.0)
        else:
            c = -s * s
        if theta_b > 0:
            c = (np.exp(theta_b * c) - 1.0) / (1.0 - np.exp(-theta_b))
        return c

    k_w = np.arange(N + 1, dtype=np.float64)
    s_w = (k_w - N) / N
    k_r = np.arange(1, N + 1, dtype=np.float64)
    s_rho = (k_r - N - 0.5) / N
    cs_w = stretch(s_w)
    cs_r = stretch(s_rho)
    s_w[0], cs_w[0] = -1.0, -1.0
    s_w[-1], cs_w[-1] = 0.0, 0.0
    return s_rho, cs_r, s_w, cs_w


def _land_mask(spec: GridSpec) -> np.ndarray:
    nx, ny = spec.xi_rho, spec.eta_rho
    mask = np.ones((nx, ny), dtype=np.int32, order="F")
    if spec.land == "corner":
        mask[:10, :10] = 0
    elif spec.land == "islands":
        rng = np.random.default_rng(spec.land_seed)
        ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
        target = spec.land_frac * nx * ny
        while (mask == 0).sum() < target:
            ci = rng.uniform(4, nx - 5)
            cj = rng.uniform(4, ny - 5)
            r = rng.uniform(1.5, 6.0)
            mask[(ii - ci) ** 2 + (jj - cj) ** 2 <= r * r] = 0
    return np.asfortranarray(mask)


def make_grid(spec: GridSpec) -> Dict[str, np.ndarray]:
    """Static grid arrays (the GRIDS(ng) fields the hot path reads)."""
    nx, ny, N = spec.xi_rho, spec.eta_rho, spec.N
    x = spec.x0 + np.arange(nx, dtype=np.float64) * spec.dx
    y = spec.y0 + np.arange(ny, dtype=np.float64) * spec.dy
    X, _ = np.meshgrid(x, y, indexing="ij")
    h = 20.0 + 180.0 * (1.0 - np.exp(-X / 30000.0))
    mask = _land_mask(spec)
    mask_u = np.asfortranarray((mask[:-1, :] * mask[1:, :]).astype(np.int32))
    mask_v = np.asfortranarray((mask[:, :-1] * mask[:, 1:]).astype(np.int32))
    s_rho, cs_r, s_w, cs_w = s_coordinate(N, spec.theta_s, spec.theta_b)
    # geographic coordinates of the rho points: a grid rotated 10 degrees
    # about (70.5 W, 41.2 N), the GRIDS(ng)%lon_rho / lat_rho of the output
    Xg, Yg = np.meshgrid(x, y, indexing="ij")
    th = math.radians(10.0)
    lat0 = 41.2
    lat = lat0 + (Xg * math.sin(th) + Yg * math.cos(th)) / 111_195.0
    lon = -70.5 + (Xg * math.cos(th) - Yg * math.sin(th)) / (111_195.0 * math.cos(math.radians(lat0)))
    return {
        "lon_rho": np.asfortranarray(lon), "lat_rho": np.asfortranarray(lat),
        "angle": np.asfortranarray(np.full((nx, ny), th)),
        "h": np.asfortranarray(h),
        "pm": np.asfortranarray(np.full((nx, ny), 1.0 / spec.dx)),
        "pn": np.asfortranarray(np.full((nx, ny), 1.0 / spec.dy)),
        "mask_rho": mask,
        "mask_u": mask_u,
        "mask_v": mask_v,
        "s_rho": s_rho, "cs_r": cs_r, "s_w": s_w, "cs_w": cs_w,
    }


def _zlevels(zeta, h, S):
    # Vtransform=2: z = zeta + (zeta + h) * S  (grid_module.f90:540)
    return zeta[..., None] + (zeta + h)[..., None] * S


def _stretch_S(h, s, cs, hc):
    return (hc * s[None, None, :] + h[..., None] * cs[None, None, :]) / (hc + h)[..., None]


def _gyre_uv(xp, yp, t, spec: GridSpec):
    """Double-gyre velocity (m/s) at physical points, time-dependent."""
    Lx = spec.gyre_lx if spec.gyre_lx else (spec.xi_rho - 1) * spec.dx
    Ly = spec.gyre_ly if spec.gyre_ly else (spec.eta_rho - 1) * spec.dy
    xs = 2.0 * xp / Lx
    ys = yp / Ly
    eps, om = 0.1, 2.0 * math.pi / (10.0 * 86400.0)
    a = eps * math.sin(om * t)
    b = 1.0 - 2.0 * a
    f = a * xs * xs + b * xs
    fx = 2.0 * a * xs + b
    psi0 = 0.3 * Ly / math.pi
    u = -psi0 * np.sin(math.pi * f) * math.pi * np.cos(math.pi * ys) / Ly
    v = psi0 * math.pi * np.cos(math.pi * f) * np.sin(math.pi * ys) * fx * (2.0 / Lx)
    if spec.eddy > 0.0:
        # submesoscale eddy field (divergence free): psi_e = A L sin(kx) sin(ky)
        k = 2.0 * math.pi / 20000.0
        u = u - spec.eddy * np.sin(k * xp) * np.cos(k * yp)
        v = v + spec.eddy * np.cos(k * xp) * np.sin(k * yp)
    return u, v


def make_frame(spec: GridSpec, grid: Dict[str, np.ndarray], t: float) -> Dict[str, np.ndarray]:
    """One hydrodynamic frame at model time ``t`` (s), HYDRODATA layout."""
    nx, ny, N = spec.xi_rho, spec.eta_rho, spec.N
    h = grid["h"]
    mask = grid["mask_rho"]
    x = spec.x0 + np.arange(nx, dtype=np.float64) * spec.dx
    y = spec.y0 + np.arange(ny, dtype=np.float64) * spec.dy
    Lx = spec.gyre_lx if spec.gyre_lx else (spec.xi_rho - 1) * spec.dx
    om = 2.0 * math.pi / M2_PERIOD
    kx = 2.0 * math.pi / max(Lx, 1.0)
    phase_r = om * t - kx * x[:, None] + 0.0 * y[None, :]
    zeta = 0.5 * np.cos(phase_r) * mask
    S_r = _stretch_S(h, grid["s_rho"], grid["cs_r"], spec.hc)
    S_w = _stretch_S(h, grid["s_w"], grid["cs_w"], spec.hc)
    z_r = _zlevels(zeta, h, S_r)
    z_w = _zlevels(zeta, h, S_w)

    # u points: between rho i and i+1
    hu = 0.5 * (h[:-1, :] + h[1:, :])
    zu = 0.5 * (z_r[:-1, :, :] + z_r[1:, :, :])
    xu = x[:-1] + 0.5 * spec.dx
    Xu, Yu = np.meshgrid(xu, y, indexing="ij")
    ug, _ = _gyre_uv(Xu, Yu, t, spec)
    ut = 0.1 * np.cos(om * t - kx * Xu)
    u = (ug[..., None] * np.exp(zu / 100.0)) + ut[..., None]
    u = u * grid["mask_u"][..., None]

    yv = y[:-1] + 0.5 * spec.dy
    Xv, Yv = np.meshgrid(x, yv, indexing="ij")
    _, vg = _gyre_uv(Xv, Yv, t, spec)
    zv = 0.5 * (z_r[:, :-1, :] + z_r[:, 1:, :])
    v = vg[..., None] * np.exp(zv / 100.0)
    v = v * grid["mask_v"][..., None]

    # w from continuity of the depth-uniform tidal current: w = -(z+h) du_t/dx
    dudx = 0.1 * kx * np.sin(om * t - kx * x[:, None]) * np.ones((1, ny))
    w = -(z_w + h[..., None]) * dudx[..., None]
    w = w * mask[..., None]

    # AKs: parabolic in depth, peak 1e-2 m^2/s, tidally modulated
    xi = (z_w + h[..., None]) / (zeta + h)[..., None]
    kmax = 1e-2 * (0.75 + 0.25 * math.cos(2.0 * om * t))
    aks = kmax * 4.0 * xi * (1.0 - xi)
    aks = np.clip(aks, 0.0, None) * mask[..., None]

    out = {"zeta": zeta, "u": u, "v": v, "w": w, "aks": aks}
    if spec.diag:
        # stratified salinity and temperature advected by the tide, and a
        # quadratic bottom stress of the bottom-level current (N/m^2 / rho0)
        tide = np.sin(om * t - kx * x[:, None])[..., None]
        out["salt"] = (33.0 + 2.0 * (1.0 - np.exp(z_r / 30.0)) + 0.3 * tide) * mask[..., None]
        out["temp"] = (8.0 + 10.0 * np.exp(z_r / 40.0) - 0.5 * tide) * mask[..., None]
        cd = 2.5e-3
        ub, vb = u[:, :, 0], v[:, :, 0]
        out["bustr"] = cd * ub * np.abs(ub)
        out["bvstr"] = cd * vb * np.abs(vb)
    if spec.behave:
        # standard deviations of turbulent acceleration (m/s^2) and vorticity
        # (1/s) decaying from the surface, and of wave acceleration (m/s^2)
        # decaying faster, tidally modulated; on the w levels
        tw = np.cos(phase_r)[..., None]
        mk = mask[..., None]
        out["turbaccel"] = 0.05 * (1.0 + 0.5 * tw) * np.exp(z_w / 20.0) * mk
        out["turbvort"] = 2.0 * (1.0 + 0.3 * tw) * np.exp(z_w / 15.0) * mk
        out["waveaccelu"] = 0.08 * (1.0 + 0.4 * tw) * np.exp(z_w / 5.0) * mk
        out["waveaccelv"] = 0.05 * (1.0 - 0.4 * tw) * np.exp(z_w / 5.0) * mk
    if spec.wetdry:
        # an intertidal flat: wet points of a coastal band go dry while the
        # tidal phase there is low; u/v masks from their rho neighbours, as
        # ROMS forms them
        Xg = x[:, None] * np.ones((1, ny))
        Yg = np.ones((nx, 1)) * y[None, :]
        Lx = (nx - 1) * spec.dx
        Ly = (ny - 1) * spec.dy
        band = (Xg > 0.3 * Lx) & (Xg < 0.7 * Lx) & (Yg > 0.25 * Ly) & (Yg < 0.75 * Ly)
        patchy = np.sin(Xg / (3.0 * spec.dx)) * np.cos(Yg / (4.0 * spec.dy)) > 0.2
        low = np.cos(phase_r) < 0.0
        dry = band & patchy & low
        wr = (mask.astype(bool) & ~dry).astype(np.float64)
        out["wetdry_rho"] = wr
        out["wetdry_u"] = wr[:-1, :] * wr[1:, :]
        out["wetdry_v"] = wr[:, :-1] * wr[:, 1:]
    if spec.stokes:
        su = 0.05 * np.exp(zu / 5.0) * math.cos(math.radians(30.0)) * grid["mask_u"][..., None]
        sv = 0.05 * np.exp(zv / 5.0) * math.sin(math.radians(30.0)) * grid["mask_v"][..., None]
        out["su"] = su
        out["sv"] = sv
    dt = np.float32 if spec.field_dtype == "f32" else np.float64
    return {k: np.asfortranarray(a.astype(np.float64 if k.startswith("wetdry") else dt)) for k, a in out.items()}


def frame_as_f64(frame: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """The frame as the reference holds it (DOUBLE PRECISION), values exact."""
    return {k: np.asfortranarray(a.astype(np.float64)) for k, a in frame.items()}


def frame_with_stokes(frame: Dict[str, np.ndarray]) -> Dict[str, np.ndarray]:
    """u += ustokes, v += vstokes in FP64, as updateHydro does under -DSTOKES
    (hydrodynamic_module.f90:606-660)."""
    f = frame_as_f64(frame)
    if "su" in f:
        f["u"] = np.asfortranarray(f["u"] + f["su"])
        f["v"] = np.asfortranarray(f["v"] + f["sv"])
    return f


def stored_frame(frame: Dict[str, np.ndarray], field_dtype: str, stokes: bool) -> Dict[str, np.ndarray]:
    """The values the device ring holds for ``frame`` (as FP64 arrays): the
    Stokes sum is formed in FP64 (as updateHydro does) and then rounded to
    the storage precision."""
    f = frame_as_f64(frame)
    if stokes and "su" in f:
        f["u"] = f["u"] + f["su"]
        f["v"] = f["v"] + f["sv"]
    out = {}
    for k in ("zeta", "u", "v", "w", "aks", "salt", "temp", "bustr", "bvstr", "wetdry_rho", "wetdry_u", "wetdry_v",
              "turbaccel", "turbvort", "waveaccelu", "waveaccelv"):
        if k not in f:
            continue
        a = f[k]
        if field_dtype == "f32":
            a = a.astype(np.float32).astype(np.float64)
        out[k] = np.asfortranarray(a)
    return out


@dataclasses.dataclass
class Release:
    """Initial particle positions in each grid's fractional index space."""
    ipos: np.ndarray   # (ngrid, n)
    jpos: np.ndarray   # (ngrid, n)
    z: np.ndarray      # (n,) initial depth (m, negative down)
    dob: np.ndarray    # (n,) release time (s)


def uniform_release(spec: GridSpec, grid, frame1, n: int, seed: int = 0,
                    dob: float = 0.0, s_range=(-0.98, -0.02)) -> Release:
    """n particles uniform in (X, Y, s) over the wet interior of one grid.

    Positions are fractional rho indices in [2, xi_rho-1) x [2, eta_rho-1),
    the range the reference's bounds() accepts (boundary_module.f90:71);
    points whose four surrounding rho points are not all wet are redrawn.
    z = zeta + (zeta + h) s with h, zeta bilinear at the point and s
    uniform over s_range: by default the column less its bottom and top
    2 %, (-1, 0) for the whole column (a well-mixed start).
    """
    rng = np.random.default_rng(seed)
    nx, ny = spec.xi_rho, spec.eta_rho
    mask = grid["mask_rho"]
    X = np.empty(n)
    Y = np.empty(n)
    filled = 0
    while filled < n:
        m = (n - filled) * 2 + 16
        xs = rng.uniform(2.0, nx - 1.0, m)
        ys = rng.uniform(2.0, ny - 1.0, m)
        I = np.floor(xs).astype(np.int64) - 1
        J = np.floor(ys).astype(np.int64) - 1
        ok = (I >= 1) & (J >= 1) & (I + 1 < nx - 1) & (J + 1 < ny - 1)
        I = np.clip(I, 0, nx - 2)
        J = np.clip(J, 0, ny - 2)
        wet = (mask[I, J] + mask[I + 1, J] + mask[I, J + 1] + mask[I + 1, J + 1]) == 4
        sel = np.nonzero(ok & wet)[0][: n - filled]
        X[filled:filled + len(sel)] = xs[sel]
        Y[filled:filled + len(sel)] = ys[sel]
        filled += len(sel)
    s = rng.uniform(s_range[0], s_range[1], n)
    I = np.floor(X).astype(np.int64)
    J = np.floor(Y).astype(np.int64)
    fx = X - I
    fy = Y - J
    I -= 1
    J -= 1

    def bil(a):
        return ((1 - fx) * (1 - fy) * a[I, J] + fx * (1 - fy) * a[I + 1, J]
                + fx * fy * a[I + 1, J + 1] + (1 - fx) * fy * a[I, J + 1])

    h = bil(grid["h"])
    zeta = bil(frame1["zeta"].astype(np.float64))
    z = zeta + (zeta + h) * s
    return Release(ipos=X[None, :].copy(), jpos=Y[None, :].copy(), z=z,
                   dob=np.full(n, dob, dtype=np.float64))


# ------------------------------------------------------------------ nesting

def nest_maps(specs: List[GridSpec]):
    """Affine index maps between every pair of grids (GRIDS(ng)%scl/off,
    grid_module.f90:441-481): X_b = scl(b)*X_a + off(b) with
    X_g = 1 + (x - x0_g)/dx_g.  Returns scl, off of shape (ngrid, ngrid, 2):
    [a][b] maps grid a's indices to grid b's.  The reference derives them
    from the first exactly coincident lon/lat point of a chain of grids;
    these are the same affine maps for any pair, siblings included."""
    ng = len(specs)
    scl = np.zeros((ng, ng, 2))
    off = np.zeros((ng, ng, 2))
    for a, A in enumerate(specs):
        for b, B in enumerate(specs):
            for c, (x0a, da, x0b, db) in enumerate(((A.x0, A.dx, B.x0, B.dx), (A.y0, A.dy, B.y0, B.dy))):
                scl[a, b, c] = da / db
                off[a, b, c] = 1.0 + (x0a - x0b - da) / db
    return scl, off


def index_of(spec: GridSpec, x: np.ndarray, y: np.ndarray):
    """Fractional rho indices of physical points in a grid."""
    return 1.0 + (x - spec.x0) / spec.dx, 1.0 + (y - spec.y0) / spec.dy


def nested_release(specs: List[GridSpec], grids, frames1, n: int, seed: int = 0,
                   child_frac: float = 0.5, dob: float = 0.0) -> Release:
    """n particles: a fraction uniform over each child's interior, the rest
    over the parent's; ipos/jpos hold each particle's indices in every grid
    (the LL2ij output of ini_ROMSPath for every grid)."""
    rng = np.random.default_rng(seed)
    parent = specs[-1]
    pg = grids[-1]
    n_child = int(n * child_frac)
    xs, ys = [], []
    kids = specs[:-1]
    per = [n_child // max(len(kids), 1)] * len(kids)
    for k, sp in enumerate(kids):
        m = per[k]
        xs.append(sp.x0 + rng.uniform(2.0, sp.xi_rho - 2.0, m) * sp.dx)
        ys.append(sp.y0 + rng.uniform(2.0, sp.eta_rho - 2.0, m) * sp.dy)
    m = n - sum(per)
    cnt = 0
    px, py = [], []
    while cnt < m:
        X = rng.uniform(2.0, parent.xi_rho - 1.0, 2 * m + 8)
        Y = rng.uniform(2.0, parent.eta_rho - 1.0, 2 * m + 8)
        I = np.floor(X).astype(int) - 1
        J = np.floor(Y).astype(int) - 1
        I = np.clip(I, 0, parent.xi_rho - 2)
        J = np.clip(J, 0, parent.eta_rho - 2)
        mk = pg["mask_rho"]
        wet = (mk[I, J] + mk[I + 1, J] + mk[I, J + 1] + mk[I + 1, J + 1]) == 4
        sel = np.nonzero(wet)[0][: m - cnt]
        px.append(parent.x0 + (X[sel] - 1.0) * parent.dx)
        py.append(parent.y0 + (Y[sel] - 1.0) * parent.dy)
        cnt += len(sel)
    x = np.concatenate(xs + px)
    y = np.concatenate(ys + py)
    ipos = np.empty((len(specs), n))
    jpos = np.empty((len(specs), n))
    for g, sp in enumerate(specs):
        ipos[g], jpos[g] = index_of(sp, x, y)
    # depth from the parent's bathymetry (same analytic h everywhere)
    s = rng.uniform(-0.95, -0.05, n)
    h = 20.0 + 180.0 * (1.0 - np.exp(-x / 30000.0))
    z = h * s
    return Release(ipos=ipos, jpos=jpos, z=z, dob=np.full(n, dob))


def batched_release(specs: List[GridSpec], grids, counts: List[int], n_ensembles: int = 16,
                    ens_min: int = 1000, ens_max: int = 500_000, seed: int = 0, ens_sigma: float = 3000.0,
                    ens_spacing_s: float = 3 * 3600.0) -> Release:
    """The batched nested release: counts[g] particles uniform over the
    interior of grid g (specs finest first, parent last; a particle released
    over the parent inside a child belongs to the child, as ini_ROMSPath's
    first-in-grid rule gives), plus n_ensembles release ensembles of
    log-uniform sizes in [ens_min, ens_max] (fixed seed): Gaussian patches
    (ens_sigma m) at random wet points of the parent, ensemble e released
    at e * ens_spacing_s.  ipos/jpos hold the indices in every grid."""
    rng = np.random.default_rng(seed)
    parent, pg = specs[-1], grids[-1]
    mk = pg["mask_rho"]

    def wet_parent(m):
        xs, ys, got = [], [], 0
        while got < m:
            X = rng.uniform(2.0, parent.xi_rho - 1.0, 2 * (m - got) + 8)
            Y = rng.uniform(2.0, parent.eta_rho - 1.0, 2 * (m - got) + 8)
            I = np.clip(np.floor(X).astype(int) - 1, 0, parent.xi_rho - 2)
            J = np.clip(np.floor(Y).astype(int) - 1, 0, parent.eta_rho - 2)
            wet = (mk[I, J] + mk[I + 1, J] + mk[I, J + 1] + mk[I + 1, J + 1]) == 4
            sel = np.nonzero(wet)[0][: m - got]
            xs.append(parent.x0 + (X[sel] - 1.0) * parent.dx)
            ys.append(parent.y0 + (Y[sel] - 1.0) * parent.dy)
            got += len(sel)
        return np.concatenate(xs), np.concatenate(ys)

    xs, ys, dobs = [], [], []
    for g, (sp, m) in enumerate(zip(specs, counts)):
        if m <= 0:
            continue
        if g == len(specs) - 1:
            x, y = wet_parent(m)
        else:
            x = sp.x0 + rng.uniform(2.0, sp.xi_rho - 2.0, m) * sp.dx
            y = sp.y0 + rng.uniform(2.0, sp.eta_rho - 2.0, m) * sp.dy
        xs.append(x)
        ys.append(y)
        dobs.append(np.zeros(m))
    sizes = np.exp(rng.uniform(np.log(ens_min), np.log(ens_max), n_ensembles)).astype(np.int64)
    cx, cy = wet_parent(n_ensembles)
    lo_x, hi_x = parent.x0 + 2.0 * parent.dx, parent.x0 + (parent.xi_rho - 2.0) * parent.dx
    lo_y, hi_y = parent.y0 + 2.0 * parent.dy, parent.y0 + (parent.eta_rho - 2.0) * parent.dy
    for e, m in enumerate(sizes):
        xs.append(np.clip(cx[e] + rng.normal(0.0, ens_sigma, m), lo_x, hi_x))
        ys.append(np.clip(cy[e] + rng.normal(0.0, ens_sigma, m), lo_y, hi_y))
        dobs.append(np.full(m, e * ens_spacing_s))
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    n = x.shape[0]
    ipos = np.empty((len(specs), n))
    jpos = np.empty((len(specs), n))
    for g, sp in enumerate(specs):
        ipos[g], jpos[g] = index_of(sp, x, y)
    s = rng.uniform(-0.95, -0.05, n)
    h = 20.0 + 180.0 * (1.0 - np.exp(-x / 30000.0))
    return Release(ipos=ipos, jpos=jpos, z=h * s, dob=np.concatenate(dobs))


# ------------------------------------------------------------------ configs

def config_spec(name: str) -> List[GridSpec]:
    """Grid specs of the named workload (one entry per grid, finest first)."""
    if name in ("cfg1", "cfg3", "cfg5"):
        return [GridSpec(130, 98, 20, land="corner", field_dtype="f64")]
    if name == "cfg2":
        return [GridSpec(512, 384, 30, land="islands", land_frac=0.08, land_seed=2,
                         stokes=True, field_dtype="f32")]
    if name == "tiny":
        return [GridSpec(24, 20, 6, land="corner", field_dtype="f64")]
    if name == "nest_tiny":
        # child (3x) inside a 40x32 parent, finest grid first
        P = GridSpec(40, 32, 6, land="corner", field_dtype="f64")
        lx, ly = (P.xi_rho - 1) * P.dx, (P.eta_rho - 1) * P.dy
        child = GridSpec(31, 25, 6, land="none", field_dtype="f64", dx=1000.0 / 3, dy=1000.0 / 3,
                         x0=14000.0, y0=9000.0, eddy=0.1, gyre_lx=lx, gyre_ly=ly)
        P.gyre_lx, P.gyre_ly = lx, ly
        return [child, P]
    if name == "nest3_tiny":
        # a parent with two sibling children, 5x (child B) and 3x (child A),
        # in config 4's [child B, child A, parent] order
        P = GridSpec(40, 32, 6, land="corner", field_dtype="f64")
        lx, ly = (P.xi_rho - 1) * P.dx, (P.eta_rho - 1) * P.dy
        A = GridSpec(31, 25, 6, land="none", field_dtype="f64", dx=1000.0 / 3, dy=1000.0 / 3,
                     x0=4000.0, y0=5000.0, eddy=0.1, gyre_lx=lx, gyre_ly=ly)
        B = GridSpec(31, 26, 6, land="none", field_dtype="f64", dx=200.0, dy=200.0,
                     x0=22000.0, y0=12000.0, eddy=0.1, gyre_lx=lx, gyre_ly=ly)
        P.gyre_lx, P.gyre_ly = lx, ly
        return [B, A, P]
    if name == "cfg4":
        # parent 400x300x30; child A 240x180x30 (3x); child B 300x250x30 (5x)
        P = GridSpec(400, 300, 30, land="islands", land_frac=0.08, land_seed=4, field_dtype="f32",
                     stokes=True)
        lx, ly = (P.xi_rho - 1) * P.dx, (P.eta_rho - 1) * P.dy
        A = GridSpec(240, 180, 30, land="none", field_dtype="f32", stokes=True, dx=1000.0 / 3, dy=1000.0 / 3,
                     x0=60000.0, y0=60000.0, eddy=0.1, gyre_lx=lx, gyre_ly=ly)
        B = GridSpec(300, 250, 30, land="none", field_dtype="f32", stokes=True, dx=200.0, dy=200.0,
                     x0=250000.0, y0=150000.0, eddy=0.1, gyre_lx=lx, gyre_ly=ly)
        P.gyre_lx, P.gyre_ly = lx, ly
        return [B, A, P]
    raise KeyError(name)


# The reference's sample behaviour settings (ROMSPath.data:56-57, 90-105,
# 123-141, 154): Process_VA/WA on, the fuchsparam values, initsize 250.
FUCHS_SAMPLE = {"process_va": 1, "process_wa": 1, "va_flag": 1, "initsize": 250.0, "swimfast": 0.0005,
                "vort_cr": 1.0, "vort_sat": 10.0, "b0pv": 0.5, "b1pv": 1.0, "b0wv": 0.0, "b1w": 0.0,
                "acc_cr": 10.0, "acc_sat": 1000.0, "b0pa": 0.5, "b1pa": 1.0, "b0wa": 0.2}


def config_params(name: str) -> dict:
    """Namelist values (ROMSPath.data groups turbparam / timeparam /
    advectparam) of the named workload."""
    base = dict(idt=300, dt=3600, scheme=1, nsb=0, vturb_on=1, hturb_on=0,
                open_ocean_boundary=0, vertdist=0.25, serr=1e-4, smth=0.6,
                sub=4.0, deltat=30.0, aksback=1e-8, constant_hturb=[0.0] * 5)
    if name == "cfg2":
        base.update(hturb_on=1, constant_hturb=[1.0] * 5)
    if name in ("tiny", "nest_tiny", "nest3_tiny"):
        base.update(hturb_on=1, constant_hturb=[1.0] * 5)
    if name == "cfg4":
        base.update(hturb_on=1, constant_hturb=[1.0] * 5)
    return base


CONFIG_PARTICLES = {"cfg1": 10_000, "cfg2": 1_048_576, "cfg3": 4_194_304,
                    "cfg5": 262_144, "tiny": 64}
# config 4: per grid (finest first: child B, child A, parent) + 16 ensembles
CONFIG4_COUNTS = [200_000, 800_000, 3_000_000]
CONFIG_DAYS = {"cfg1": 2.0, "cfg2": 10.0, "cfg3": 10.0, "cfg4": 5.0, "cfg5": 3.0, "tiny": 0.25}
