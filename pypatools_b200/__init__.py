"""pypatools_b200: B200 (sm_100a) particle pusher with fused trilinear E/B
field-map interpolation, a drop-in for PyPATools' ``Pusher`` hot path.

    from pypatools_b200 import Pusher, Field, IonSpecies
    pusher = Pusher(IonSpecies('proton'), 'boris')              # float64, the drop-in
    r_hist, v_hist, active = pusher.track_batch(r0, v0, efield, bfield, nsteps, dt)
    fast = Pusher(IonSpecies('proton'), 'boris', precision='mixed')

The kernels live in ``lib/libppt.so`` (build: ``python -m pypatools_b200.build``).
"""
from .species import IonSpecies, PRESETS
from .field import Field, ScaledField, CompositeField, FieldMap, get_interpolator, CudaInterpolator
from .pusher import Pusher, PusherGPU, RFModulation, DeviceTracker
from .particles import ParticleDistribution
from .moments import bunch_moments
from .deposit import bin_particles_cic
from .electrodes import ElectrodeSurface
from .beam import Beam

__all__ = ["IonSpecies", "PRESETS", "Field", "ScaledField", "CompositeField", "FieldMap", "get_interpolator",
           "CudaInterpolator", "Pusher", "PusherGPU", "RFModulation", "DeviceTracker", "ParticleDistribution",
           "bunch_moments", "bin_particles_cic", "ElectrodeSurface", "Beam"]
