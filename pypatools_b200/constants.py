"""Physical constants used on the pusher path.

The values come from ``scipy.constants`` exactly as the reference's
``src/PyPATools/global_variables.py:35-43`` takes them, so that
``q_over_m``, the light-speed clamps and the v <-> beta*gamma conversions are
bit-identical to the reference's.
"""
from scipy import constants as _const

CLIGHT = _const.speed_of_light
ECHARGE = _const.elementary_charge
AMU_MEV = _const.value("atomic mass constant energy equivalent in MeV")
EMASS_MEV = _const.value("electron mass energy equivalent in MeV")
PMASS_MEV = _const.value("proton mass energy equivalent in MeV")
MUMASS_MEV = _const.value("muon mass energy equivalent in MeV")

# global_variables.py:33 -- floor used for the x' = vx/vz angle denominators
EPSILON = 1e-10

# Settings.txt defaults the reference ships with (settings.py:33-37):
# relativistic v <-> beta*gamma conversion, energy from |p| (not pz alone).
RELATIVISTIC = True
Z_ENERGY = False

# Clamp used by every relativistic kernel of the reference
# (pusher.py:93-94 for beta^2, pusher.py:276, 359, 615, 888 for |v|).
BETA_SQ_CLAMP = 0.9999
V_CLAMP_FRACTION = 0.9999
