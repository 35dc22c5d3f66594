"""``Beam``: the snapshot store of a tracking run (src/PyPATools/beam.py:20-296).

Positions, velocities and alive flags of every particle at the save points
(every ``save_freq`` steps, ``n_saves = ceil(n_steps / save_freq)``), and the
time of each, with the reference's methods: ``set_pd_at_step``,
``get_pd_at_step`` / ``_at_index`` / ``_at_time``, ``find_nearest_step``,
``get_nearest_pd``, ``get_time_array``, ``get_n_saves``,
``reset_save_counter``.  ``Beam.from_track`` fills one from the histories and
``active`` mask of ``PusherGPU.track_batch`` (numpy arrays or the device
tensors of ``snapshot='device'``).

The reference's class does not run as written: its constructor passes
``n_particles`` to ``ParticleDistribution`` (which takes no such argument),
``set_pd_at_step`` reads ``pd.alive`` (the attribute is ``alive_mask``) and
``get_pd_at_index`` assigns (N, 3) arrays to the 1-D ``x`` view and calls a
``copy`` method that does not exist (beam.py:87-90, :133, :281-288).  This
class stores and returns what those lines mean to: a NEW
``ParticleDistribution`` per call, built from the saved positions and
velocities (beta*gamma from v as ``set_p_from_v_vec`` does) with the saved
alive mask.
"""
import numpy as np

from .particles import ParticleDistribution


class Beam:
    def __init__(self, species, n_particles, n_steps, save_freq):
        if save_freq < 1:
            raise ValueError("save_freq must be >= 1")
        self.species = species
        self.n_particles = int(n_particles)
        self.n_steps = int(n_steps)
        self.save_freq = int(save_freq)
        self.n_saves = (self.n_steps + self.save_freq - 1) // self.save_freq
        self.t = np.full(self.n_saves, np.nan)
        self.x_vec = np.full((self.n_saves, self.n_particles, 3), np.nan)
        self.v_vec = np.full((self.n_saves, self.n_particles, 3), np.nan)
        self.alive = np.zeros((self.n_saves, self.n_particles), dtype=bool)
        self._current_save_idx = 0

    @classmethod
    def from_track(cls, species, r_hist, v_hist, active, nsteps, dt, rec_every_n_steps=1, t0=0.0):
        """The records of one ``track_batch`` call: record k is step
        k * rec_every_n_steps (n_steps = nsteps + 1, so the final record is a
        save point).  A particle is alive at a record while its row there is
        finite; ``active`` (False = stopped by an electrode) marks the end."""
        def host(a):
            return a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
        r, v = host(r_hist), host(v_hist)
        n_rec, m, _ = r.shape
        beam = cls(species, m, int(nsteps) + 1, rec_every_n_steps)
        k = min(n_rec, beam.n_saves)
        beam.t[:k] = t0 + np.arange(k) * rec_every_n_steps * dt
        beam.x_vec[:k] = r[:k]
        beam.v_vec[:k] = v[:k]
        beam.alive[:k] = np.isfinite(r[:k]).all(axis=2)
        if active is not None and k == n_rec:
            # a particle stopped at the last step was recorded there, then stopped
            beam.alive[k - 1] &= host(active).astype(bool)
        beam._current_save_idx = k
        return beam

    def _save_index(self, step):
        if step % self.save_freq != 0:
            raise ValueError(f"Timestep {step} is not a save point. "
                             f"Only multiples of save_freq={self.save_freq} are saved.")
        return step // self.save_freq

    def set_pd_at_step(self, pd, step, time):
        """Copy a ParticleDistribution's positions, velocities and alive mask
        into the save point of ``step`` (beam.py:95-134)."""
        idx = self._save_index(step)
        if idx >= self.n_saves:
            raise IndexError(f"Timestep {step} → save index {idx}, exceeds n_saves={self.n_saves}")
        self.t[idx] = time
        self.x_vec[idx] = pd.x_vec
        self.v_vec[idx] = pd.v_vec
        self.alive[idx] = pd.alive_mask

    def get_pd_at_step(self, step):
        return self.get_pd_at_index(self._save_index(step))

    def get_pd_at_time(self, time):
        hits = np.nonzero(self.t == time)[0]
        if hits.size == 0:
            raise ValueError(f"Time {time} not found in saved times. "
                             "Use find_nearest_step() for approximate matches.")
        return self.get_pd_at_index(int(hits[0]))

    def find_nearest_step(self, target_time):
        # among the save points that were set (the reference's argmin would
        # return an unset, NaN-time save point first)
        idx = int(np.nanargmin(np.abs(self.t - target_time)))
        return idx * self.save_freq, self.t[idx]

    def get_nearest_pd(self, target_time):
        step, _ = self.find_nearest_step(target_time)
        return self.get_pd_at_step(step)

    def get_pd_at_index(self, index):
        """A new ParticleDistribution for save index ``index`` (negative
        indices count from the end)."""
        if index < 0:
            index = self.n_saves + index
        if not 0 <= index < self.n_saves:
            raise IndexError(f"Save index {index} out of range [0, {self.n_saves})")
        pd = ParticleDistribution(species=self.species, x_vec=self.x_vec[index].copy(),
                                  p_vec=np.zeros((self.n_particles, 3)), recalculate=False)
        pd.set_p_from_v_vec(self.v_vec[index])
        pd.alive_mask = self.alive[index].copy()
        pd.t = self.t[index]
        return pd

    def get_time_array(self):
        return self.t.copy()

    def get_n_saves(self):
        return self.n_saves

    def reset_save_counter(self):
        self._current_save_idx = 0
