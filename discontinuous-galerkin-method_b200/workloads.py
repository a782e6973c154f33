"""Synthetic workloads: meshes, media, sources and receivers of the benchmark configurations.

Every workload is fully determined by its seeds.  Sizes follow the five configurations the
engine is measured on (homogeneous square, coupled acoustic-elastic slope, heterogeneous
random medium, multi-shot layered batch, uneven multi-mesh batch) plus small meshes used as
parity fixtures.  The reference fixes the Ricker peak frequency and the sponge geometry at
compile time (dg.h:5, 8-12); a workload carries them as data.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import meshgen


@dataclasses.dataclass
class Workload:
    name: str
    mesh: meshgen.Mesh
    vp: np.ndarray            # (K,) m/s
    vs: np.ndarray            # (K,) m/s (0 in fluid elements)
    rho: np.ndarray           # (K,) kg/m^3
    fp: float                 # Ricker peak frequency, Hz (dg.h:5)
    sponge: tuple             # (bound_x, bound_z, model_w, model_h), metres (dg.h:8-12)
    src: np.ndarray           # (S, 2) source vertex positions, one per shot
    rec: np.ndarray           # (R, 2) receiver vertex positions
    steps: int
    beta: float = 0.1         # sponge taper strength (DG_leap_Frog_OpenMP.c:300)
    pi: float = 3.1415        # the reference's Pi (dg.h:6), used by the wavelet and sponge

    @property
    def K(self) -> int:
        return self.mesh.K

    @property
    def shots(self) -> int:
        return int(self.src.shape[0])

    def dof_per_step(self) -> int:
        """DOF-updates per time step: 5 fields x 6 nodes per element and shot."""
        return 30 * self.K * self.shots

    def materials(self) -> np.ndarray:
        return np.stack([self.vp, self.vs, self.rho], 1).astype(np.float64)


def gardner(vp):
    return 310.0 * np.asarray(vp, dtype=np.float64) ** 0.25


def poly_model(poly, materials: dict, src, rec, *, h=None, fp=15.0, sponge=None, steps=2000, seed=0) -> Workload:
    """A model from a ``.poly`` planar straight-line graph (path or text; input_files/mesh/*.poly
    are of this kind): triangulated by ``meshgen.from_poly``, region attribute ``a`` getting
    ``materials[a] = (vp, vs, rho)`` (vs = 0: fluid), sources and receivers moved to the nearest
    vertex.  ``sponge`` = (bound_x, bound_z, model_w, model_h) in absolute coordinates (dg.h:8-12);
    default: a band of 5 % of the extent inside the bounding box.  The reference assigns
    materials from the attributes in its driver (DG_leap_Frog_OpenMP.c:248-262)."""
    mesh = meshgen.from_poly(poly, h, seed=seed)
    table = {int(k): v for k, v in materials.items()}
    missing = sorted(set(np.unique(mesh.attr).tolist()) - set(table))
    if missing:
        raise ValueError("no material for region attributes %s" % missing)
    mat = np.array([table[int(a)] for a in mesh.attr], dtype=np.float64)
    if sponge is None:
        lo, hi = mesh.points.min(0), mesh.points.max(0)
        b = 0.05 * (hi - lo)
        sponge = (lo[0] + b[0], lo[1] + b[1], hi[0] - lo[0] - 2 * b[0], hi[1] - lo[1] - 2 * b[1])
    if sponge[0] <= 0 or sponge[1] <= 0:
        raise ValueError("the sponge box must start at positive coordinates (bound_x, bound_z > 0)")
    return Workload("poly_model_K%d" % mesh.K, mesh, mat[:, 0], mat[:, 1], mat[:, 2], float(fp), tuple(sponge),
                    meshgen.snap_to_vertices(mesh, src), meshgen.snap_to_vertices(mesh, rec), int(steps))


def homogeneous_square(n_cells=100, size=2000.0, steps=2000, seed=0, n_rec=101, shots=1) -> Workload:
    """2 km x 2 km square, n x n cells split in two, interior vertices jittered +-10% h."""
    centre = (size / 2, size / 2)
    h = size / n_cells
    srcs = [centre]
    if shots > 1:
        srcs = [(round((size * (i + 1) / (shots + 1)) / h) * h, centre[1]) for i in range(shots)]
    mesh = meshgen.jittered_grid(n_cells, n_cells, size, size, jitter=0.1, seed=seed, pinned=srcs)
    K = mesh.K
    rx = np.linspace(0.0, size, n_rec)
    rx = np.round(rx / h) * h
    rec = np.stack([rx, np.full_like(rx, size)], 1)
    b = 100.0
    return Workload("homogeneous_square_K%d" % K, mesh, np.full(K, 3000.0), np.full(K, 1732.0),
                    np.full(K, 2000.0), 15.0, (b, b, size - 2 * b, size - 2 * b),
                    meshgen.snap_to_vertices(mesh, srcs), meshgen.snap_to_vertices(mesh, rec), steps)


def coupled_slope(width=6000.0, height=3000.0, h=10.0, steps=6000, seed=2, n_rec=301,
                  amp=200.0, wavelength=1500.0) -> Workload:
    """Coupled acoustic-elastic model under a sinusoidal top surface (Delaunay of jittered points).

    Water layer (vs = 0, vp = 1500, rho = 1000) below the surface, three elastic layers with
    vp 2500/3200/4000, vs = vp/sqrt(3), rho from Gardner's relation.
    """
    ztop0 = height - amp
    top = lambda x: ztop0 + amp * np.sin(2 * np.pi * np.asarray(x, dtype=np.float64) / wavelength)  # noqa: E731
    src = (width / 2, round(height * 0.4 / h) * h)
    rx = np.round(np.linspace(0.0, width, n_rec) / h) * h
    rec = np.stack([rx, top(rx)], 1)
    mesh = meshgen.delaunay(width, height, h, seed=seed, top=top, pinned=[src])
    cz = mesh.centroids()[:, 1]
    vp = np.where(cz > 0.7 * height, 1500.0, np.where(cz > 0.45 * height, 2500.0,
                                                       np.where(cz > 0.2 * height, 3200.0, 4000.0)))
    fluid = vp == 1500.0
    vs = np.where(fluid, 0.0, vp / math.sqrt(3.0))
    rho = np.where(fluid, 1000.0, gardner(vp))
    b = 100.0
    return Workload("coupled_slope_K%d" % mesh.K, mesh, vp, vs, rho, 20.0,
                    (b, b, width - 2 * b, height - 2 * b), meshgen.snap_to_vertices(mesh, [src]),
                    meshgen.snap_to_vertices(mesh, rec), steps)


def gaussian_random_field(shape, spacing, corr_len, seed):
    """Stationary Gaussian field with Gaussian covariance, unit variance, on a regular grid."""
    rng = np.random.default_rng(seed)
    ny, nx = shape
    white = rng.standard_normal(shape)
    kx = np.fft.fftfreq(nx, d=spacing) * 2 * np.pi
    ky = np.fft.fftfreq(ny, d=spacing) * 2 * np.pi
    kk = kx[None, :] ** 2 + ky[:, None] ** 2
    amp = np.exp(-kk * corr_len ** 2 / 8.0)
    field = np.real(np.fft.ifft2(np.fft.fft2(white) * amp))
    field -= field.mean()
    field /= field.std()
    return field


def random_medium(width=10000.0, height=5000.0, n_cells_x=1000, n_cells_z=1000, steps=10000,
                  seed=1, n_rec=501, mean_vp=3500.0, rel_std=0.10, corr_len=200.0) -> Workload:
    """Heterogeneous elastic medium with a log-normal Gaussian-random-field vp per element."""
    hx = width / n_cells_x
    hz = height / n_cells_z
    src = (round(width / 2 / hx) * hx, round(height * 0.5 / hz) * hz)
    mesh = meshgen.jittered_grid(n_cells_x, n_cells_z, width, height, jitter=0.1, seed=seed,
                                 pinned=[src])
    g = 10.0
    field = gaussian_random_field((int(height / g) + 1, int(width / g) + 1), g, corr_len, seed)
    cen = mesh.centroids()
    ix = np.clip(np.round(cen[:, 0] / g).astype(int), 0, field.shape[1] - 1)
    iz = np.clip(np.round(cen[:, 1] / g).astype(int), 0, field.shape[0] - 1)
    sig = math.sqrt(math.log(1 + rel_std ** 2))
    mu = math.log(mean_vp) - 0.5 * sig ** 2
    vp = np.exp(mu + sig * field[iz, ix])
    vs = vp / 1.8
    rho = gardner(vp)
    rx = np.round(np.linspace(0.0, width, n_rec) / hx) * hx
    rec = np.stack([rx, np.full_like(rx, height)], 1)
    b = 100.0
    return Workload("random_medium_K%d" % mesh.K, mesh, vp, vs, rho, 25.0,
                    (b, b, width - 2 * b, height - 2 * b), meshgen.snap_to_vertices(mesh, [src]),
                    meshgen.snap_to_vertices(mesh, rec), steps)


def layered_multishot(nx=400, nz=250, h=20.0, shots=64, steps=4000, seed=3, n_rec=201,
                      shot_phase: float = 0.0) -> Workload:
    """Layered elastic mesh (K = 2 nx nz), ``shots`` sources evenly spaced 200 m below the top.

    ``shot_phase`` in [0, 1) shifts every source along the surface by that fraction of the
    shot spacing (a different shot set on the same mesh)."""
    width, height = nx * h, nz * h
    zsrc = height - 200.0
    xs = [round(width * (i + 0.5 + shot_phase) / shots / h) * h for i in range(shots)]
    srcs = [(x, zsrc) for x in xs]
    mesh = meshgen.jittered_grid(nx, nz, width, height, jitter=0.1, seed=seed, pinned=srcs)
    cz = mesh.centroids()[:, 1]
    vp = np.where(cz > 0.75 * height, 2000.0, np.where(cz > 0.4 * height, 3000.0, 4000.0))
    vs = vp / math.sqrt(3.0)
    rho = gardner(vp)
    rx = np.round(np.linspace(0.0, width, n_rec) / h) * h
    rec = np.stack([rx, np.full_like(rx, height)], 1)
    b = 100.0
    return Workload("layered_multishot_K%d_S%d" % (mesh.K, shots), mesh, vp, vs, rho, 15.0,
                    (b, b, width - 2 * b, height - 2 * b), meshgen.snap_to_vertices(mesh, srcs),
                    meshgen.snap_to_vertices(mesh, rec), steps)


def uneven_batch(n_meshes=48, kmin=5000, kmax=500000, seed=5, t_end=1.5):
    """48 independent meshes, K log-uniform in [kmin, kmax], random layered vp, 1-8 shots.

    All meshes cover the same 2 km x 2 km square, so a finer mesh takes a smaller dt; every
    mesh runs ceil(t_end / dt) steps (dt from the reference formula, set on the host).
    """
    rng = np.random.default_rng(seed)
    out = []
    size = 2000.0
    for m in range(n_meshes):
        K = float(np.exp(rng.uniform(np.log(kmin), np.log(kmax))))
        n = max(4, int(round(math.sqrt(K / 2))))
        h = size / n
        shots = int(rng.integers(1, 9))
        xs = [round(size * (i + 1) / (shots + 1) / h) * h for i in range(shots)]
        zsrc = round(size * 0.8 / h) * h
        srcs = [(x, zsrc) for x in xs]
        mesh = meshgen.jittered_grid(n, n, size, size, jitter=0.1, seed=seed * 1000 + m,
                                     pinned=srcs)
        nl = int(rng.integers(2, 5))
        vps = np.sort(rng.uniform(1500.0, 4500.0, size=nl))
        cz = mesh.centroids()[:, 1]
        layer = np.clip(((size - cz) / size * nl).astype(int), 0, nl - 1)
        vp = vps[layer]
        vs = vp / math.sqrt(3.0)
        rho = gardner(vp)
        rx = np.round(np.linspace(0.0, size, 41) / h) * h
        rec = np.stack([rx, np.full_like(rx, size)], 1)
        b = 100.0
        out.append(Workload("uneven_%02d_K%d_S%d" % (m, mesh.K, shots), mesh, vp, vs, rho, 15.0,
                            (b, b, size - 2 * b, size - 2 * b), meshgen.snap_to_vertices(mesh, srcs),
                            meshgen.snap_to_vertices(mesh, rec), 0))
    return out, t_end


# --- small meshes that the parity fixtures are made from -----------------------------------

def small_square(n_cells=12, steps=200, shots=1, seed=0) -> Workload:
    w = homogeneous_square(n_cells=n_cells, steps=steps, seed=seed, n_rec=n_cells + 1, shots=shots)
    w.name = "small_square_K%d_S%d" % (w.K, shots)
    return w


def small_slope(h=150.0, steps=200, seed=7) -> Workload:
    """Coupled acoustic-elastic Delaunay mesh on 2 km x 1.5 km with a curved top."""
    width, height = 2000.0, 1500.0
    top = lambda x: 1400.0 + 100.0 * np.sin(2 * np.pi * np.asarray(x, dtype=np.float64) / 1000.0)  # noqa: E731
    src = (1050.0, 600.0)
    mesh = meshgen.delaunay(width, height, h, seed=seed, top=top, pinned=[src])
    cz = mesh.centroids()[:, 1]
    vp = np.where(cz > 1000.0, 1500.0, np.where(cz > 500.0, 2500.0, 3500.0))
    fluid = vp == 1500.0
    vs = np.where(fluid, 0.0, vp / math.sqrt(3.0))
    rho = np.where(fluid, 1000.0, gardner(vp))
    rx = np.linspace(0.0, width, 11)
    rec = np.stack([rx, top(rx)], 1)
    return Workload("small_slope_K%d" % mesh.K, mesh, vp, vs, rho, 15.0, (100.0, 100.0, 1800.0, 1300.0),
                    meshgen.snap_to_vertices(mesh, [src]), meshgen.snap_to_vertices(mesh, rec), steps)
