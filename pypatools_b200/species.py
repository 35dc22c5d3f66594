"""Ion species: the only thing the pusher path reads from it is ``q_over_m``.

Mirrors the reference's ``IonSpecies`` (src/PyPATools/species.py:39-187) so
that scripts written against the reference keep working.  The pusher accepts
ANY object that has a ``q_over_m`` attribute (and ``name`` for ``repr``), the
reference's own ``IonSpecies`` included.

Parity note: the reference computes the rest mass as ``a * AMU_MEV``
(species.py:117) and ignores the preset's ``mass_mev`` (read at :80).  A
proton's q/m is therefore not CODATA's e/m_p.  This class keeps that exact
formula so q/m matches the reference bit for bit.
"""
from .constants import AMU_MEV, ECHARGE, CLIGHT, EMASS_MEV, PMASS_MEV, MUMASS_MEV

# Preset table (species.py:7-36).  The numbers must be the reference's for
# q/m to agree; the table layout is this module's own.
PRESETS = {
    "proton":   dict(a=1.00727647, z=1.0, q=1.0, mass_mev=PMASS_MEV, latex=r"$\mathrm{p}^+$"),
    "H_1-":     dict(a=1.00837361135, z=1.0, q=1.0, mass_mev=1.00837361135 * AMU_MEV, latex=r"$\mathrm{H}^1-$"),
    "electron": dict(a=EMASS_MEV / AMU_MEV, z=0.0, q=-1.0, mass_mev=EMASS_MEV, latex=r"$\mathrm{e}^-$"),
    "muon":     dict(a=MUMASS_MEV / AMU_MEV, z=0.0, q=-1.0, mass_mev=MUMASS_MEV, latex=r"$\mu^-$"),
    "H2_1+":    dict(a=2.01533, z=2.0, q=1.0, mass_mev=2.01533 * AMU_MEV, latex=r"$\mathrm{H}_2^+$"),
    "4He_2+":   dict(a=4.001506179127, z=2.0, q=2.0, mass_mev=4.001506179127 * AMU_MEV, latex=r"$^4\mathrm{He}^{2+}$"),
}


class IonSpecies:
    """Charge/mass holder with the reference's constructor and properties."""

    def __init__(self, name, label=None, latex_label=None, a=None, z=None, q=None):
        if name in PRESETS:
            preset = PRESETS[name]
            a, z, q = preset["a"], preset["z"], preset["q"]
            if latex_label is None:
                latex_label = preset["latex"]
        elif None in (a, z, q):
            # The reference prints and calls exit(1) here (species.py:93-97);
            # a library should raise instead of killing the interpreter.
            raise ValueError(f"ion species {name!r} needs a, z and q (got a={a}, z={z}, q={q})")
        self._name = name
        self._label = name if label is None else label
        self._latex_label = name if latex_label is None else latex_label
        self._a = a
        self._z = z
        self._q = q
        self._mass_mev = a * AMU_MEV
        self._mass_kg = self._mass_mev * ECHARGE * 1.0e6 / CLIGHT ** 2.0

    @property
    def name(self):
        return self._name

    @property
    def label(self):
        return self._label

    @property
    def latex_label(self):
        return self._latex_label

    @property
    def a(self):
        return self._a

    @property
    def q(self):
        return self._q

    @property
    def charge(self):
        return self._q * ECHARGE

    @property
    def mass_mev(self):
        return self._mass_mev

    @property
    def mass_kg(self):
        return self._mass_kg

    @property
    def mass_electron_multiple(self):
        return self._mass_mev / EMASS_MEV

    @property
    def mass_opera(self):
        return self._mass_mev / EMASS_MEV

    @property
    def q_over_a(self):
        return self._q / self._a

    @property
    def q_over_m(self):
        """Charge-to-mass ratio in C/kg, the scalar every pusher kernel uses."""
        return self._q * ECHARGE / self._mass_kg

    def __str__(self):
        return (f"Ion Species {self._name} with label {self._label}:\n"
                f"A = {self._a}, Z = {self._z}, q = {self._q}\n"
                f"M_0 = {self._mass_mev} MeV/c^2 = {self._mass_kg} kg, Q = {self._q * ECHARGE} C")
