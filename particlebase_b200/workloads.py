"""Seeded synthetic LJ systems in reduced units (sigma = epsilon = m = kB = 1).

These stand in for the reference drivers' hand-built initial states
(testMD2.cu:14-85 builds a lattice and Maxwell-Boltzmann velocities from
std::mt19937): the reference ships no datasets, so every workload here is
generated from a seed with the shapes and distributions of the benchmark
configurations.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class LJSystem:
    """One periodic LJ system in host memory (particle order)."""

    box: np.ndarray            # (6,) float32: xmin, xmax, ymin, ymax, zmin, zmax
    r: np.ndarray              # (N, 3) float64 positions inside the box
    v: np.ndarray              # (N, 3) float64 velocities
    mass: np.ndarray           # (N,) float64
    types: np.ndarray          # (N,) uint32 type ids
    lj: np.ndarray             # (ntypes, ntypes, 3) float64: sigma, epsilon, rc per pair
    rc: float                  # cell-grid cutoff (largest pair cutoff)
    temperature: float = 1.0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return len(self.r)

    @property
    def ntypes(self) -> int:
        return self.lj.shape[0]

    @property
    def L(self) -> np.ndarray:
        b = self.box.astype(np.float64)
        return np.array([b[1] - b[0], b[3] - b[2], b[5] - b[4]])


def single_type_lj(rc: float = 2.5) -> np.ndarray:
    return np.array([[[1.0, 1.0, rc]]])


def kob_andersen_lj() -> np.ndarray:
    """Kob-Andersen 80:20 parameters with per-pair cutoff 2.5 sigma_ab."""
    sig = np.array([[1.0, 0.8], [0.8, 0.88]])
    eps = np.array([[1.0, 1.5], [1.5, 0.5]])
    return np.stack([sig, eps, 2.5 * sig], axis=-1)


def fcc_positions(cells: int, density: float):
    """fcc lattice of cells^3 unit cells x 4 sites at the given number density.

    Sites (0,0,0), (1/2,1/2,0), (1/2,0,1/2), (0,1/2,1/2) times a, with
    a = (4/rho)^(1/3) adjusted so that cells * a is exactly the FP32 box length
    (the lattice is then exactly periodic in the box the device holds); the
    lattice is shifted by a/4 so no site lies on a face.
    Returns (positions (N,3) float64, box length L).
    """
    a = (4.0 / density) ** (1.0 / 3.0)
    a = float(np.float32(a * cells)) / cells
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(cells)
    ijk = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 1, 3)
    pos = ((ijk + basis[None]) * a + 0.25 * a).reshape(-1, 3)
    return pos, a * cells


def maxwell_boltzmann(n: int, temperature: float, rng: np.random.Generator, mass=None):
    """Normal velocities with zero total momentum, rescaled to exactly T.

    The rescale uses T = sum m v^2 / (3 N kB), the reference's calcTemp
    (cudaParticleMD.hh:89-92).
    """
    mass = np.ones(n) if mass is None else mass
    v = rng.normal(0.0, 1.0, (n, 3)) * np.sqrt(temperature / mass)[:, None]
    v -= (mass[:, None] * v).sum(0) / mass.sum()
    t = (mass[:, None] * v * v).sum() / (3 * n)
    v *= np.sqrt(temperature / t)
    return v


def fcc_system(cells: int, density: float, temperature: float, seed: int,
               rc: float = 2.5, name: str = "") -> LJSystem:
    pos, L = fcc_positions(cells, density)
    rng = np.random.default_rng(seed)
    n = len(pos)
    v = maxwell_boltzmann(n, temperature, rng)
    box = np.array([0, L, 0, L, 0, L], np.float32)
    # positions as the device will hold them (float32), inside [0, L)
    pos = np.mod(pos, np.float64(box[1]))
    return LJSystem(box=box, r=pos, v=v, mass=np.ones(n), types=np.zeros(n, np.uint32),
                    lj=single_type_lj(rc), rc=rc, temperature=temperature,
                    name=name or f"fcc{cells}", meta={"density": density, "seed": seed})


def config_c1(seed: int = 1) -> LJSystem:
    """4,000 atoms, fcc 10^3 x 4, rho 0.8442, T* 0.72, rc 2.5 (NVE)."""
    return fcc_system(10, 0.8442, 0.72, seed, name="lj_fcc_4000_nve")


def config_c2(seed: int = 2) -> LJSystem:
    """1,048,576 atoms, fcc 64^3 x 4, rho 0.8442, T* 0.72, rc 2.5 (Gaussian)."""
    return fcc_system(64, 0.8442, 0.72, seed, name="lj_fcc_1048576_gauss")


def kob_andersen_random(n: int, density: float, temperature: float, seed: int) -> LJSystem:
    """80:20 Kob-Andersen mixture at uniform random positions (to be relaxed)."""
    rng = np.random.default_rng(seed)
    L = (n / density) ** (1.0 / 3.0)
    box = np.array([0, L, 0, L, 0, L], np.float32)
    pos = rng.uniform(0.0, float(box[1]), (n, 3))
    pos = np.minimum(pos, np.nextafter(np.float32(box[1]), np.float32(0)).astype(np.float64))
    types = np.zeros(n, np.uint32)
    types[rng.permutation(n)[: n // 5]] = 1
    v = maxwell_boltzmann(n, temperature, rng)
    lj = kob_andersen_lj()
    return LJSystem(box=box, r=pos, v=v, mass=np.ones(n), types=types, lj=lj,
                    rc=float(lj[..., 2].max()), temperature=temperature,
                    name=f"ka_{n}", meta={"density": density, "seed": seed})


def config_c5(seed: int = 5, n: int = 8_388_608) -> LJSystem:
    return kob_andersen_random(n, 1.2, 0.8, seed)


def fcc_cells_for(n_target: float) -> int:
    """Nearest k with 4 k^3 atoms to n_target (k >= 5)."""
    k = max(5, int(round((n_target / 4.0) ** (1.0 / 3.0))))
    return k


def uneven_replicas(count: int = 256, n_lo: float = 500, n_hi: float = 50_000,
                    rho=(0.70, 0.90), temp=(0.7, 1.5), seed: int = 3,
                    rc: float = 2.5) -> list[LJSystem]:
    """Independent fcc replicas with N log-uniform in [n_lo, n_hi] rounded to 4k^3."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n_target = float(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        k = fcc_cells_for(n_target)
        d = float(rng.uniform(*rho))
        t = float(rng.uniform(*temp))
        s = fcc_system(k, d, t, seed=int(rng.integers(1 << 31)), rc=rc, name=f"replica{i}")
        out.append(s)
    return out


@dataclass
class JobSpec:
    """One served MD job: arrival time (s), fcc cells k (4 k^3 atoms), density,
    temperature, step count and the seed of its velocities."""

    arrival: float
    cells: int
    density: float
    temperature: float
    steps: int
    seed: int

    @property
    def n(self) -> int:
        return 4 * self.cells ** 3

    def system(self, rc: float = 2.5) -> LJSystem:
        return fcc_system(self.cells, self.density, self.temperature, self.seed, rc=rc,
                          name=f"job_{self.seed}")


def served_jobs(count: int = 2000, rate: float = 50.0, n_lo: float = 1_000, n_hi: float = 200_000,
                rho=(0.75, 0.90), temp=(0.7, 1.2), steps=(100, 5_000),
                seed: int = 4) -> list[JobSpec]:
    """Poisson arrival stream of LJ jobs: exponential gaps of mean 1/rate,
    N log-uniform in [n_lo, n_hi] rounded to a 4k^3 fcc count, density and T*
    uniform, step count uniform over the integers in `steps`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        n_target = float(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))
        out.append(JobSpec(arrival=t, cells=fcc_cells_for(n_target),
                           density=float(rng.uniform(*rho)), temperature=float(rng.uniform(*temp)),
                           steps=int(rng.integers(steps[0], steps[1] + 1)),
                           seed=int(rng.integers(1 << 31))))
    return out
