"""``Beam``, the snapshot store (src/PyPATools/beam.py:20-296).

The reference's class cannot be constructed as written (its constructor
passes ``n_particles`` to ``ParticleDistribution``, beam.py:87-90), so these
tests check the behaviour its code and docstrings describe: save points every
``save_freq`` steps, ceil(n_steps / save_freq) of them, NaN-initialised
arrays, the errors for non-save steps and out-of-range indices, and new
ParticleDistribution objects on every get."""
import numpy as np
import pytest

from pypatools_b200 import Beam, IonSpecies
from pypatools_b200.particles import ParticleDistribution, momenta_from_velocities


def _pd(rng, m):
    x = rng.normal(0, 1e-3, (m, 3))
    v = rng.normal(0, 1e5, (m, 3)) + np.array([0, 0, 1.4e7])
    pd = ParticleDistribution(species=IonSpecies("proton"), x_vec=x, p_vec=momenta_from_velocities(v),
                              recalculate=False)
    return pd, x, v


def test_save_points_and_round_trip():
    rng = np.random.default_rng(1)
    beam = Beam(IonSpecies("proton"), 50, n_steps=1001, save_freq=100)
    assert beam.get_n_saves() == 11 and np.isnan(beam.x_vec).all() and not beam.alive.any()
    pd, x, v = _pd(rng, 50)
    pd.alive_mask[3] = False
    beam.set_pd_at_step(pd, 300, 3e-9)
    with pytest.raises(ValueError):
        beam.set_pd_at_step(pd, 301, 0.0)
    with pytest.raises(IndexError):
        beam.set_pd_at_step(pd, 1100, 0.0)
    out = beam.get_pd_at_step(300)
    np.testing.assert_array_equal(out.x_vec, x)
    np.testing.assert_allclose(out.v_vec, v, rtol=1e-15)
    assert not out.alive_mask[3] and out.alive_mask.sum() == 49
    out.x_vec[:] = 0.0                     # a copy: the store is unchanged
    np.testing.assert_array_equal(beam.x_vec[3], x)
    assert beam.find_nearest_step(2.9e-9) == (300, 3e-9)
    np.testing.assert_array_equal(beam.get_pd_at_time(3e-9).x_vec, x)
    with pytest.raises(ValueError):
        beam.get_pd_at_time(1.0)
    with pytest.raises(IndexError):
        beam.get_pd_at_index(11)
    assert np.isnan(beam.get_pd_at_index(-1).x_vec).all()


def test_from_track_histories():
    rng = np.random.default_rng(2)
    n_rec, m = 5, 7
    r = rng.normal(size=(n_rec, m, 3))
    v = rng.normal(size=(n_rec, m, 3))
    r[3:, 2] = np.nan                       # stopped after record 2
    v[3:, 2] = np.nan
    active = np.ones(m, dtype=bool)
    active[2] = active[5] = False           # particle 5 stopped on the last step, recorded there
    beam = Beam.from_track(IonSpecies("proton"), r, v, active, nsteps=400, dt=1e-10, rec_every_n_steps=100)
    assert beam.n_saves == n_rec
    np.testing.assert_allclose(beam.get_time_array(), np.arange(5) * 1e-8)
    assert beam.alive[2, 2] and not beam.alive[3, 2] and beam.alive[3, 5] and not beam.alive[4, 5]
    np.testing.assert_array_equal(beam.get_pd_at_step(200).x_vec, r[2])
