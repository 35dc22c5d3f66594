"""``ParticleDistribution`` with the reference's boundary API, moments on the GPU.

Keeps what the pusher path touches (src/PyPATools/particles.py:123-788):
(N,3) position / beta*gamma storage, the per-component v <-> beta*gamma
conversions the reference uses (particles.py:71-117, :393-457; relativistic
settings), kinetic energies, and the collective statistics (centroid, rms
sizes, x-x' correlations, emittances, energy mean / spread), which are
computed by the ``ppt_moments`` kernel in float64.
"""
import numpy as np

from .constants import CLIGHT, EPSILON
from .moments import bunch_moments
from .species import IonSpecies


def velocities_from_momenta(p):
    """Per-component beta*gamma -> v (particles.py:71-91)."""
    p = np.asarray(p, dtype=np.float64)
    return CLIGHT * p / np.sqrt(p ** 2 + 1.0)


def momenta_from_velocities(v):
    """Per-component v -> beta*gamma with the 0.99999 c^2 clamp (particles.py:94-117)."""
    v = np.asarray(v, dtype=np.float64)
    v_sq = np.where(v ** 2 >= CLIGHT ** 2, 0.99999 * CLIGHT ** 2, v ** 2)
    return v / np.sqrt(CLIGHT ** 2 - v_sq)


class ParticleDistribution:
    def __init__(self, species=None, x=None, y=None, z=None, px=None, py=None, pz=None, x_vec=None, p_vec=None,
                 q=0.0, f=0.0, recalculate=True):
        self._species = species if species is not None else IonSpecies("proton")
        separate = any(a is not None for a in (x, y, z, px, py, pz))
        vector = x_vec is not None or p_vec is not None
        if separate and vector:
            raise ValueError("Cannot specify both separate coordinates (x,y,z,px,py,pz) AND vector "
                             "coordinates (x_vec, p_vec). Choose one method.")
        if vector:
            if x_vec is None or p_vec is None:
                raise ValueError("Both x_vec and p_vec must be provided together.")
            x_vec, p_vec = np.asarray(x_vec, dtype=np.float64), np.asarray(p_vec, dtype=np.float64)
            if x_vec.shape != p_vec.shape:
                raise ValueError(f"x_vec and p_vec must have same shape. Got x_vec: {x_vec.shape}, "
                                 f"p_vec: {p_vec.shape}")
            if x_vec.ndim != 2 or x_vec.shape[1] != 3:
                raise ValueError(f"x_vec and p_vec must have shape (N, 3). Got: {x_vec.shape}")
            self._x_vec, self._p_vec = x_vec.copy(), p_vec.copy()
        else:
            cols = [np.zeros(1) if a is None else np.asarray(a, dtype=np.float64) for a in (x, y, z, px, py, pz)]
            if len({len(c) for c in cols}) != 1:
                raise ValueError("All coordinate arrays must have same length.")
            self._x_vec = np.column_stack(cols[:3])
            self._p_vec = np.column_stack(cols[3:])
        self.q, self.f = q, f
        self.numpart = len(self._x_vec)
        self.alive_mask = np.ones(self.numpart, dtype=bool)
        self._stats = None
        if recalculate:
            self.recalculate_all()

    # -- storage -------------------------------------------------------------
    @property
    def species(self):
        return self._species

    @property
    def x_vec(self):
        return self._x_vec

    @x_vec.setter
    def x_vec(self, value):
        value = np.asarray(value, dtype=np.float64)
        if value.shape != self._x_vec.shape:
            raise ValueError(f"Positions must have shape {self._x_vec.shape}, got {value.shape}")
        self._x_vec = value.copy()
        self._stats = None

    @property
    def p_vec(self):
        return self._p_vec

    @p_vec.setter
    def p_vec(self, value):
        value = np.asarray(value, dtype=np.float64)
        if value.shape != self._p_vec.shape:
            raise ValueError(f"Momenta must have shape {self._p_vec.shape}, got {value.shape}")
        self._p_vec = value.copy()
        self._stats = None

    @property
    def v_vec(self):
        return velocities_from_momenta(self._p_vec)

    def set_p_from_v_vec(self, v_vec):
        self._p_vec = momenta_from_velocities(v_vec)
        self._stats = None

    def set_p_from_v(self, vx, vy, vz):
        self.set_p_from_v_vec(np.column_stack([vx, vy, vz]))

    @property
    def x(self):
        return self._x_vec[:, 0]

    @property
    def y(self):
        return self._x_vec[:, 1]

    @property
    def z(self):
        return self._x_vec[:, 2]

    @property
    def px(self):
        return self._p_vec[:, 0]

    @property
    def py(self):
        return self._p_vec[:, 1]

    @property
    def pz(self):
        return self._p_vec[:, 2]

    @property
    def xp_vec(self):
        v = self.v_vec
        vz = np.where(np.abs(v[:, 2]) < 1e-10, EPSILON, v[:, 2])
        return v / vz[:, None]

    @property
    def ekin_mev(self):
        pr = np.linalg.norm(self._p_vec, axis=1)
        m = self._species.mass_mev
        return m * pr ** 2 / (1.0 + np.sqrt(1.0 + pr ** 2))

    # -- collective properties (GPU) ------------------------------------------
    def _moments(self):
        if self._stats is None:
            self._stats = bunch_moments(self._x_vec, self.v_vec, self._species.mass_mev)
        return self._stats

    def recalculate_all(self):
        self.numpart = len(self._x_vec)
        self._stats = None
        if self.numpart:
            self._moments()

    def calculate_centroid(self):
        return self._moments()["centroid"]

    def calculate_stdevs(self):
        return self._moments()["x_std"]

    @property
    def centroid(self):
        return self._moments()["centroid"]

    @property
    def mean_momentum_betagamma(self):
        return self._moments()["mean_p"]

    @property
    def mean_energy_mev(self):
        return self._moments()["ekin_mean"]

    @property
    def rms_energy_spread_mev(self):
        return self._moments()["ekin_std"]

    @property
    def x_std(self):
        return self._moments()["x_std"][0]

    @property
    def y_std(self):
        return self._moments()["x_std"][1]

    @property
    def z_std(self):
        return self._moments()["x_std"][2]

    def get_emittances(self, normalized=True):
        st = self._moments()
        return st["emittance_n"] if normalized else st["emittance"]

    def get_beam_edges(self, mode="1rms"):
        st = self._moments()
        if mode == "1rms":
            lo, hi = st["centroid"] - st["x_std"], st["centroid"] + st["x_std"]
        elif mode == "2rms":
            lo, hi = st["centroid"] - 2.0 * st["x_std"], st["centroid"] + 2.0 * st["x_std"]
        elif mode == "full":
            lo, hi = self._x_vec.min(axis=0), self._x_vec.max(axis=0)
        else:
            raise ValueError(f"Unknown mode: {mode}. Use '1rms', '2rms', or 'full'")
        return np.column_stack((lo, hi)).flatten()
