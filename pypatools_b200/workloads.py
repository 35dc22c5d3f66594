"""Seeded synthetic workloads for the pusher hot path.

The reference publishes no datasets or field maps for this path, so every
workload is synthetic: a seeded bunch (``numpy.random.default_rng(seed)``,
float64) and an analytic field map sampled on a uniform node grid.  The same
function feeds the tests, the golden-fixture script and ``bench.py``, so the
GPU and the CPU oracle always see identical float64 inputs.

Workloads (sizes are the defaults; every function accepts smaller ``n`` /
``nsteps`` for parity cases):

* ``quad_solenoid_protons``   4096 protons, 0.9-1.1 MeV, 65^3 B map over
  +-5 cm (Bz = 1 T plus a 10 T/m quadrupole), E = 0, dt = 1e-11 s, 1000 steps.
* ``radial_e_solenoid_electrons``  1e6 electrons, 10 keV-10 MeV log-uniform,
  isotropic, 129^3 E+B map over +-10 cm (E radial 1 MV/m at r = 0.1 m,
  Bz = 0.5 T cos(pi z / 0.2 m)), dt = 1e-12 s, 1e4 steps.
* ``rf_gap_protons``  1e7 protons, 1 MeV +-1 %, 256^3 float32 E+B map over a
  20 cm cube (Ez = 5 MV/m sin(pi (z + 0.1) / 0.2), Bz = 0.2 T), E modulated by
  cos(2 pi 100 MHz t + phi_i), dt = 1e-11 s, 2e4 steps, snapshot every 500.
* ``sector_ring_protons``  1e8 protons, 5 MeV +-0.5 %, 512^3 float32 B map
  over a 1 m cube (Bz = 1 T (1 + 0.1 cos 4 theta) - 0.05 T/m r), E = 0,
  dt = 1e-10 s, 5e4 steps.
"""
from dataclasses import dataclass, field
from typing import Optional, Dict, Tuple

import numpy as np

from .constants import CLIGHT
from .species import IonSpecies


@dataclass
class Workload:
    name: str
    species: IonSpecies
    r0: np.ndarray                      # (M, 3) float64 [m]
    v0: np.ndarray                      # (M, 3) float64 [m/s]
    grid: Tuple[np.ndarray, np.ndarray, np.ndarray]
    e_values: Optional[Dict[str, np.ndarray]]   # {'x','y','z'} -> (nx,ny,nz) or None (E = 0)
    b_values: Optional[Dict[str, np.ndarray]]
    dt: float
    nsteps: int
    rec_every: int
    rf_frequency: Optional[float] = None
    rf_phase: Optional[np.ndarray] = None       # (M,) float64 [rad]
    meta: dict = field(default_factory=dict)

    @property
    def n(self):
        return self.r0.shape[0]


def _beam_velocity(ke_mev, direction, mass_mev):
    """|v| = beta c from kinetic energy, along unit ``direction`` rows."""
    gamma = 1.0 + ke_mev / mass_mev
    beta = np.sqrt(1.0 - 1.0 / gamma ** 2)
    return direction * (beta * CLIGHT)[:, None]


def _unit_rows(d):
    return d / np.linalg.norm(d, axis=1)[:, None]


def _materialise(a, shape, dtype):
    return np.ascontiguousarray(np.broadcast_to(a, shape), dtype=dtype)


def quad_solenoid_protons(n=4096, nsteps=1000, seed=0, nodes=65, rec_every=1):
    rng = np.random.default_rng(seed)
    ion = IonSpecies("proton")
    ke = rng.uniform(0.9, 1.1, n)
    thx = rng.normal(0.0, 5e-3, n)
    thy = rng.normal(0.0, 5e-3, n)
    d = _unit_rows(np.stack([np.tan(thx), np.tan(thy), np.ones(n)], axis=1))
    v0 = _beam_velocity(ke, d, ion.mass_mev)
    r0 = rng.uniform(-0.01, 0.01, (n, 3))
    g = np.linspace(-0.05, 0.05, nodes)
    shape = (nodes,) * 3
    gy = g[None, :, None]
    gx = g[:, None, None]
    b = {"x": _materialise(10.0 * gy, shape, np.float64),
         "y": _materialise(10.0 * gx, shape, np.float64),
         "z": np.ones(shape, dtype=np.float64)}
    return Workload("quad_solenoid_protons", ion, r0, v0, (g, g.copy(), g.copy()), None, b,
                    dt=1e-11, nsteps=nsteps, rec_every=rec_every)


def radial_e_solenoid_electrons(n=1_000_000, nsteps=10_000, seed=2, nodes=129, rec_every=None,
                                map_dtype=np.float64):
    rng = np.random.default_rng(seed)
    ion = IonSpecies("electron")
    ke = 10.0 ** rng.uniform(np.log10(0.01), np.log10(10.0), n)
    d = _unit_rows(rng.normal(size=(n, 3)))
    v0 = _beam_velocity(ke, d, ion.mass_mev)
    r0 = rng.normal(0.0, 2e-3, (n, 3))
    g = np.linspace(-0.1, 0.1, nodes)
    shape = (nodes,) * 3
    gx, gy, gz = g[:, None, None], g[None, :, None], g[None, None, :]
    e = {"x": _materialise(1e7 * gx, shape, map_dtype),
         "y": _materialise(1e7 * gy, shape, map_dtype),
         "z": np.zeros(shape, dtype=map_dtype)}
    b = {"x": np.zeros(shape, dtype=map_dtype),
         "y": np.zeros(shape, dtype=map_dtype),
         "z": _materialise(0.5 * np.cos(np.pi * gz / 0.2), shape, map_dtype)}
    return Workload("radial_e_solenoid_electrons", ion, r0, v0, (g, g.copy(), g.copy()), e, b,
                    dt=1e-12, nsteps=nsteps, rec_every=rec_every or nsteps)


def rf_gap_protons(n=10_000_000, nsteps=20_000, seed=3, nodes=256, rec_every=500,
                   map_dtype=np.float32, frequency=1e8):
    rng = np.random.default_rng(seed)
    ion = IonSpecies("proton")
    ke = 1.0 * rng.uniform(0.99, 1.01, n)
    x = rng.normal(0.0, 1e-3, n)
    y = rng.normal(0.0, 1e-3, n)
    xp = rng.normal(0.0, 2e-3, n)
    yp = rng.normal(0.0, 2e-3, n)
    d = _unit_rows(np.stack([xp, yp, np.ones(n)], axis=1))
    v0 = _beam_velocity(ke, d, ion.mass_mev)
    v_nom = _beam_velocity(np.array([1.0]), np.array([[0.0, 0.0, 1.0]]), ion.mass_mev)[0, 2]
    half = 0.5 * v_nom / frequency          # bunch spans one RF period of flight
    z = rng.uniform(-half, half, n)
    phase = rng.uniform(0.0, 2.0 * np.pi, n)
    r0 = np.stack([x, y, z], axis=1)
    g = np.linspace(-0.1, 0.1, nodes)
    shape = (nodes,) * 3
    gz = g[None, None, :]
    e = {"x": np.zeros(shape, dtype=map_dtype),
         "y": np.zeros(shape, dtype=map_dtype),
         "z": _materialise(5e6 * np.sin(np.pi * (gz + 0.1) / 0.2), shape, map_dtype)}
    b = {"x": np.zeros(shape, dtype=map_dtype),
         "y": np.zeros(shape, dtype=map_dtype),
         "z": np.full(shape, 0.2, dtype=map_dtype)}
    return Workload("rf_gap_protons", ion, r0, v0, (g, g.copy(), g.copy()), e, b,
                    dt=1e-11, nsteps=nsteps, rec_every=rec_every,
                    rf_frequency=frequency, rf_phase=phase)


def sector_ring_equilibrium_radius(ion, ke_mev):
    """Radius where p/(q Bz) closes with the azimuthal average Bz = 1 - 0.05 r."""
    m = ion.mass_mev
    p_mev = np.sqrt(ke_mev ** 2 + 2.0 * ke_mev * m)
    b_rho = p_mev * 1e6 / CLIGHT / abs(ion.q)
    # r (1 - 0.05 r) = b_rho  ->  0.05 r^2 - r + b_rho = 0, small root
    return (1.0 - np.sqrt(1.0 - 4.0 * 0.05 * b_rho)) / (2.0 * 0.05)


def sector_ring_bz(x, y):
    r = np.hypot(x, y)
    th = np.arctan2(y, x)
    return 1.0 * (1.0 + 0.1 * np.cos(4.0 * th)) - 0.05 * r


def sector_ring_protons(n=100_000_000, nsteps=50_000, seed=5, nodes=512, rec_every=None,
                        map_dtype=np.float32):
    rng = np.random.default_rng(seed)
    ion = IonSpecies("proton")
    ke = 5.0 * rng.uniform(0.995, 1.005, n)
    r_eq = sector_ring_equilibrium_radius(ion, 5.0)
    dx = rng.normal(0.0, 3e-3, n)
    dy = rng.normal(0.0, 3e-3, n)
    dz = rng.normal(0.0, 3e-3, n)
    xr = rng.normal(0.0, 3e-3, n)          # radial angle
    zr = rng.normal(0.0, 3e-3, n)          # vertical angle
    # Momentum along -y: a positive charge in +Bz then circulates clockwise
    # about the origin, so the orbit stays inside the +-0.5 m map.
    d = _unit_rows(np.stack([xr, -np.ones(n), zr], axis=1))
    v0 = _beam_velocity(ke, d, ion.mass_mev)
    r0 = np.stack([r_eq + dx, dy, dz], axis=1)
    g = np.linspace(-0.5, 0.5, nodes)
    shape = (nodes,) * 3
    bz2 = sector_ring_bz(g[:, None], g[None, :])
    b = {"x": None, "y": None,
         "z": _materialise(bz2[:, :, None].astype(map_dtype), shape, map_dtype)}
    return Workload("sector_ring_protons", ion, r0, v0, (g, g.copy(), g.copy()), None, b,
                    dt=1e-10, nsteps=nsteps, rec_every=rec_every or nsteps,
                    meta={"r_eq": r_eq})


def serving_maps(map_dtype=np.float32):
    """The 4 resident maps of the serving stream: 64^3 quadrupole-solenoid B
    (+-5 cm), 128^3 radial E + solenoid B (+-10 cm), 192^3 and 256^3 RF-gap
    Ez + Bz (+-10 cm, static).  Returns [(grid, e_values, b_values), ...]."""
    out = []
    q = quad_solenoid_protons(n=1, nsteps=1, nodes=64)
    out.append((q.grid, None, {c: q.b_values[c].astype(map_dtype) for c in "xyz"}))
    r = radial_e_solenoid_electrons(n=1, nsteps=1, nodes=128, map_dtype=map_dtype)
    out.append((r.grid, r.e_values, r.b_values))
    for nodes in (192, 256):
        g = rf_gap_protons(n=1, nsteps=1, nodes=nodes, map_dtype=map_dtype)
        out.append((g.grid, g.e_values, g.b_values))
    return out


@dataclass
class ServingJobSpec:
    job_id: int
    arrival: float
    n: int
    algorithm: str
    nsteps: int
    map_index: int
    r0: np.ndarray
    v0: np.ndarray


def serving_stream(n_jobs=2000, rate=50.0, seed=4, n_min=1e3, n_max=1e6, steps_min=1000, steps_max=10000,
                   algorithms=("boris", "vay_rel", "rk4_rel"), n_maps=4):
    """Poisson arrivals at ``rate`` jobs/s; particle counts log-uniform in
    [n_min, n_max]; pusher uniform over ``algorithms``; step counts uniform
    in [steps_min, steps_max]; map uniform over the resident maps; each bunch
    drawn like the quadrupole-solenoid protons with seed 1000 + job_id."""
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_jobs))
    ns = np.exp(rng.uniform(np.log(n_min), np.log(n_max), n_jobs)).astype(np.int64)
    algs = rng.integers(0, len(algorithms), n_jobs)
    steps = rng.integers(steps_min, steps_max + 1, n_jobs)
    maps = rng.integers(0, n_maps, n_jobs)
    specs = []
    for j in range(n_jobs):
        b = quad_solenoid_protons(n=int(ns[j]), nsteps=int(steps[j]), seed=1000 + j, nodes=2)
        specs.append(ServingJobSpec(j, float(arrivals[j]), int(ns[j]), algorithms[int(algs[j])], int(steps[j]),
                                    int(maps[j]), b.r0, b.v0))
    return specs
