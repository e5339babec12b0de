"""Synthetic workloads in the reference's input-deck format.

Every deck is a binary Al-Cu alloy: C0 = 4.5 wt%, liquidus slope -2.6 K/wt%,
k = 0.14, D_l = 3e-9 m^2/s, D_s = 3e-13 m^2/s, Gibbs-Thomson 2.4e-7 K m.
The liquidus is 933.47 K (pure Al melting point, an assumed physical
constant) + m C0; the solidus T_m + m C0 / k.

Time step: the reference's explicit update keeps ce >= 0 only while
3 D_l dt / dx^2 < k (a fully solid cell, cl = ce / k, next to liquid
cells); with k = 0.14 every deck here uses D_l dt / dx^2 = 0.04.
"""
from __future__ import annotations

import numpy as np

T_MELT = 933.47
C0, SLOPE, K_PART = 4.5, -2.6, 0.14
D_LIQ, D_SOL, GIBBS = 3e-9, 3e-13, 2.4e-7
T_LIQ = T_MELT + SLOPE * C0
T_SOL = T_MELT + SLOPE * C0 / K_PART
FOURIER = 0.04  # D_l dt / dx^2


def quat_to_rotmat(q) -> np.ndarray:
    """Row-major 3x3 rotation matrix of a (w, x, y, z) quaternion (normalised here)."""
    w, x, y, z = np.asarray(q, dtype=np.float64) / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def random_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform on SO(3) (Shoemake's subgroup algorithm, three uniforms per quaternion)."""
    u = rng.random((n, 3))
    a, b = np.sqrt(1 - u[:, 0]), np.sqrt(u[:, 0])
    return np.stack([a * np.sin(2 * np.pi * u[:, 1]), a * np.cos(2 * np.pi * u[:, 1]),
                     b * np.sin(2 * np.pi * u[:, 2]), b * np.cos(2 * np.pi * u[:, 2])], 1)


def _alloy_deck(name: str, dims, dx: float, *, tip_curv: int, t0: float, gradient: float, velocity: float,
                cooling: float, rho_v: float, mu: float, sigma: float, rho_s: float, max_grains: int,
                seed: int, extra: str = "") -> str:
    dt = FOURIER * dx * dx / D_LIQ
    return f"""BaseFileName {name}
NSubblocks 1 1 1
NCellsPerSB {dims[0]} {dims[1]} {dims[2]}
FaceCtrl 1 1 1 1 1 1
CellSize {dx!r}
FSGrow 0.66
TimeStep {dt!r}
RandSeedVal {seed}
TipCurvature {tip_curv}
GibbsThomsonCoef {GIBBS!r}
FinishTime 0
FsFinish 1.1
LiquidusTemp {T_LIQ!r}
SolidusTemp {T_SOL!r}
Cinit {C0!r}
m_solute0 0 0 {SLOPE!r}
part_coef0 0 0 {K_PART!r}
Dsol {D_SOL!r}
Dliq {D_LIQ!r}
InitialTemperature {t0!r}
Gradient {gradient!r}
Velocity {velocity!r}
CoolingRate {cooling!r}
ScreenPFreq 0
MaxGrainDensity {rho_v!r}
GNGaussCentre {mu!r}
GNGaussSigma {sigma!r}
MaxGrainDensitySurf {rho_s!r}
GNGaussCentreSurf {mu!r}
GNGaussSigmaSurf {sigma!r}
MaxTotGrains {max_grains}
GNOriented 1
{extra}"""


def one_grain(n: int = 64, dx: float = 1e-6, tip_curv: int = 1) -> tuple[str, np.ndarray, np.ndarray, np.ndarray]:
    """One seed at the domain centre in a uniformly cooled melt: uniform
    temperature starting at the liquidus, 50 K/s, zero-flux faces, seed
    threshold 0 (nucleates on the first step below the liquidus), its
    orientation the quaternion drawn from seed 0; no other site.

    Returns (deck text, site cells (1 x 3, 0-based), thresholds, rotmats (1 x 9))."""
    deck = _alloy_deck(f"onegrain{n}", (n, n, n), dx, tip_curv=tip_curv, t0=T_LIQ, gradient=0.0, velocity=0.0,
                       cooling=50.0, rho_v=0.0, mu=2.0, sigma=0.5, rho_s=0.0, max_grains=16, seed=0)
    cells = np.array([[n // 2, n // 2, n // 2]], dtype=np.int32)
    thr = np.zeros(1, dtype=np.float32)
    rot = quat_to_rotmat(random_quaternions(np.random.default_rng(0), 1)[0]).reshape(1, 9)
    return deck, cells, thr, rot


def setup_one_grain(dom, cells, thr, rot) -> None:
    dom.set_sites(cells, thr)
    dom.set_site_orientations(cells, rot)


def am_track(dims=(512, 256, 128), dx: float = 1e-6, seed: int = 3) -> str:
    """Single-track AM melt pool: the reference's moving-source quadrature
    (AnalyticalThermal 1, temperature.c:62-123; not the closed-form
    Rosenthal solution) at 0.5 m/s, 150 W, absorptivity 0.4, k_th 100 W/m/K
    and rho c_p = k_th / alpha = 3.33e6 J/m^3/K (alpha 3e-5 m^2/s).  Spot
    diameter 50 um, start 50 um before the domain at mid-width, substrate top
    8 um below the domain top, substrate at 300 K.  Bulk sites 1e14 m^-3
    with undercooling N(3 K, 1 K).  Spot size, start and substrate
    temperature are this workload's own choices."""
    nx, ny, nz = dims
    extra = f"""AnalyticalThermal 1
LaserPower 150
LaserSpeed 0.5
LaserSpotSize 50e-6
LaserAbsorption 0.4
LaserHatchSpacing 50e-6
LaserStartLocation {-50e-6!r} {ny * dx / 2!r} {(nz - 8) * dx!r}
NoOfLayers 1
SubInitialTemp 300
ThermalConductivity 100
SpecificHeat 395
Density {100 / 3e-5 / 395!r}
"""
    return _alloy_deck(f"am{nx}", dims, dx, tip_curv=0, t0=300.0, gradient=0.0, velocity=0.0, cooling=0.0,
                       rho_v=1e14, mu=3.0, sigma=1.0, rho_s=0.0, max_grains=1000000, seed=seed, extra=extra)


def columnar_columns(gx: int, gy: int, dx: float, mean_width: float = 20e-6, seed: int = 11):
    """Grain id of every (x, y) column of a columnar substrate: a Voronoi
    tessellation of the x-y plane with one seed per mean_width^2, ids 1..n;
    and the n grains' rotation matrices (row-major, random orientations).
    Returns (cols (gy x gx int32), rotmats (n x 9))."""
    rng = np.random.default_rng(seed)
    n = max(1, int(round(gx * gy * dx * dx / (mean_width * mean_width))))
    sx = rng.uniform(0, gx, n)
    sy = rng.uniform(0, gy, n)
    yy, xx = np.mgrid[0:gy, 0:gx]
    px, py = xx.ravel() + 0.5, yy.ravel() + 0.5
    best = np.zeros(px.size, dtype=np.int32)
    bd = np.full(px.size, np.inf)
    for s in range(n):
        d = (px - sx[s]) ** 2 + (py - sy[s]) ** 2
        m = d < bd
        bd[m] = d[m]
        best[m] = s
    cols = (best + 1).reshape(gy, gx).astype(np.int32)
    rot = np.stack([quat_to_rotmat(q).ravel() for q in random_quaternions(rng, n)])
    return cols, rot


def columnar_substrate(shape_zyx, dx: float, top_plane: int, mean_width: float = 20e-6, seed: int = 11):
    """Columnar grains filling interior planes 1..top_plane (see
    columnar_columns).  Returns (gr, rotmats (n x 9)) with gr in the halo'd
    layout (int32, zeros outside the substrate)."""
    nz, ny, nx = shape_zyx
    cols, rot = columnar_columns(nx - 2, ny - 2, dx, mean_width, seed)
    gr = np.zeros(shape_zyx, dtype=np.int32)
    gr[1:top_plane + 1, 1:-1, 1:-1] = cols[None]
    return gr, rot


def write_substrate_file(path, cols: np.ndarray, rot: np.ndarray, top_plane: int) -> None:
    """The same substrate for the reference, in the format its harness reads
    (MMSREF_INJECT_SUBSTRATE of oracle/ref_shim/ref_hooks.c): int32 gx, gy,
    top, n; int32 cols[gy][gx]; f64 rot[n][9]."""
    gy, gx = cols.shape
    with open(path, "wb") as f:
        f.write(np.array([gx, gy, top_plane, len(rot)], dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(cols, dtype="<i4").tobytes())
        f.write(np.ascontiguousarray(rot, dtype="<f8").tobytes())


def setup_substrate(dom, top_plane: int, dx: float, mean_width: float = 20e-6, seed: int = 11) -> int:
    """Pre-fills a domain with columnar substrate grains (fs = 1); returns their number."""
    gr0 = dom.download("gr")
    gr, rot = columnar_substrate(gr0.shape, dx, top_plane, mean_width, seed)
    fs = dom.download("fs")
    fs[gr > 0] = 1.0
    dom.set_grains(rot)
    dom.upload("gr", gr)
    dom.upload("fs", fs)
    return len(rot)


def ensemble(n: int = 64, seed: int = 2026, edges=(32, 48, 64, 96, 128), dx: float = 1e-6) -> list[str]:
    """Independent solidification domains: edges drawn uniformly from
    `edges` per axis, cooling rate log-uniform in 10-1000 K/s from the
    liquidus, bulk nucleation density log-uniform in 1e11-1e14 m^-3 with
    undercooling N(2 K, 0.5 K), each with its own random seed."""
    rng = np.random.default_rng(seed)
    decks = []
    for d in range(n):
        dims = tuple(int(rng.choice(edges)) for _ in range(3))
        rate = float(10 ** rng.uniform(1, 3))
        rho = float(10 ** rng.uniform(11, 14))
        decks.append(_alloy_deck(f"ens{d}", dims, dx, tip_curv=0, t0=T_LIQ, gradient=0.0, velocity=0.0,
                                 cooling=rate, rho_v=rho, mu=2.0, sigma=0.5, rho_s=0.0, max_grains=100000,
                                 seed=int(rng.integers(1, 2 ** 31 - 1))))
    return decks
