"""Generate the golden fixtures in this folder by running the reference.

The reference (DanielWinklehner/PyPATools) is pure Python + Numba and has no
golden vectors or tests for the pusher path, so parity is pinned by running
its own ``Pusher.track_batch`` / ``Pusher.track`` / ``Field`` /
``ParticleDistribution`` code on seeded inputs and storing the results.

Run from the repository root, with PYPATOOLS_REFERENCE_SRC naming the
reference checkout's ``src`` directory (it is only needed to regenerate; the
fixtures are committed):

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python tests/golden/make_golden.py

Import shims: ``pusher.py:33`` imports ``py_electrodes`` unconditionally and
the package imports ``h5py`` and ``matplotlib`` at module level; none of them
is on the path, so inert stub modules stand in for them.  The package also
``rmtree``s ``./temp`` at import (``global_variables.py:27-29``), so the import
runs from a scratch working directory, and Numba's cache goes to /tmp because
the source tree is read-only.
"""
import os
import sys
import tempfile
import types
from pathlib import Path

import numpy as np


def reference_src():
    """The reference checkout's ``src`` directory, from PYPATOOLS_REFERENCE_SRC."""
    src = os.environ.get("PYPATOOLS_REFERENCE_SRC")
    if not src or not (Path(src) / "PyPATools" / "pusher.py").is_file():
        raise SystemExit("set PYPATOOLS_REFERENCE_SRC to the reference checkout's src directory "
                         "(the one holding PyPATools/pusher.py)")
    return src

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def load_reference():
    os.environ.setdefault("NUMBA_CACHE_DIR", os.path.join(tempfile.gettempdir(), "ppt_ref_numba"))

    class _Stub(types.ModuleType):
        __path__ = []

        def __getattr__(self, key):
            if key.startswith("__"):
                raise AttributeError(key)
            sub = sys.modules.get(f"{self.__name__}.{key}")
            return sub if sub is not None else type(key, (), {})

    for name in ["py_electrodes", "py_electrodes.py_electrodes", "h5py", "matplotlib",
                 "matplotlib.pyplot", "matplotlib.cm", "matplotlib.colors", "matplotlib.ticker"]:
        sys.modules.setdefault(name, _Stub(name))
    cwd = os.getcwd()
    os.chdir(tempfile.mkdtemp(prefix="ppt_ref_"))
    sys.path.insert(0, reference_src())
    try:
        from PyPATools import pusher, field, species, particles
    finally:
        os.chdir(cwd)
    return pusher, field, species, particles


def main():
    sys.path.insert(0, str(REPO))
    from pypatools_b200 import workloads

    pusher, field, species, particles = load_reference()
    Pusher, Field = pusher.Pusher, field.Field
    out = {}

    def ref_field(grid, values):
        if values is None:
            return Field.zero(dim=3)
        g = {"x": grid[0], "y": grid[1], "z": grid[2]}
        return Field.from_arrays(g, {c: np.asarray(values[c], dtype=np.float64) for c in "xyz"})

    # -- species q/m (species.py:117-163) ------------------------------------
    for name in sorted(species.PRESETS):
        out[f"species/{name}/q_over_m"] = np.float64(species.IonSpecies(name).q_over_m)

    # -- quad-solenoid protons, full size, Boris (the reference's own CPU case)
    wl = workloads.quad_solenoid_protons()
    ef, bf = ref_field(wl.grid, wl.e_values), ref_field(wl.grid, wl.b_values)
    qm = wl.species.q_over_m
    rh, vh, act = Pusher(wl.species, "boris").track_batch(wl.r0, wl.v0, ef, bf, 1000, wl.dt, 500)
    out.update({"c1/r0": wl.r0, "c1/v0": wl.v0, "c1/q_over_m": np.float64(qm),
                "c1/boris/r_hist": rh, "c1/boris/v_hist": vh, "c1/boris/active": act})
    # the other reference algorithms on a 256-particle subsample
    sub = slice(0, 4096, 16)
    for alg in ["leapfrog", "rk4", "yoshida", "vay_rel", "rk4_rel", "yoshida_rel"]:
        rh, vh, _ = Pusher(wl.species, alg).track_batch(wl.r0[sub], wl.v0[sub], ef, bf, 1000, wl.dt, 250)
        out[f"c1/{alg}/r_hist"] = rh
        out[f"c1/{alg}/v_hist"] = vh
        print("c1", alg, "done")

    # -- radial-E / solenoid electrons: 128-particle subsample, 1e4 steps ----
    wl2 = workloads.radial_e_solenoid_electrons(n=128)
    ef2, bf2 = ref_field(wl2.grid, wl2.e_values), ref_field(wl2.grid, wl2.b_values)
    out.update({"c2/r0": wl2.r0, "c2/v0": wl2.v0})
    for alg in ["boris", "vay_rel", "rk4_rel"]:
        rh, vh, _ = Pusher(wl2.species, alg).track_batch(wl2.r0, wl2.v0, ef2, bf2, 10000, wl2.dt, 2500)
        out[f"c2/{alg}/r_hist"] = rh
        out[f"c2/{alg}/v_hist"] = vh
        print("c2", alg, "done")

    # -- interpolation edge cases (interpolators.py:88-135) -------------------
    rng = np.random.default_rng(11)
    gx = np.linspace(-0.05, 0.05, 9)
    gy = np.sort(np.concatenate([[-0.04, 0.06], rng.uniform(-0.04, 0.06, 9)]))   # non-uniform
    gz = np.linspace(0.0, 0.3, 7)
    vals = {c: rng.normal(size=(gx.size, gy.size, gz.size)) for c in "xyz"}
    probe = np.concatenate([
        np.stack([rng.uniform(-0.06, 0.06, 400), rng.uniform(-0.05, 0.07, 400),
                  rng.uniform(-0.05, 0.35, 400)], axis=1),
        # exactly on the faces, on interior nodes, one ulp outside
        np.array([[gx[0], gy[0], gz[0]], [gx[-1], gy[-1], gz[-1]], [gx[3], gy[4], gz[2]],
                  [np.nextafter(gx[-1], 1), 0.0, 0.1], [np.nextafter(gx[0], -1), 0.0, 0.1],
                  [0.0, gy[-1], gz[-1]], [0.0, 0.0, np.nextafter(gz[0], -1)]]),
    ])
    fmap = Field.from_arrays({"x": gx, "y": gy, "z": gz}, vals)
    out.update({"interp/gx": gx, "interp/gy": gy, "interp/gz": gz, "interp/probe": probe,
                "interp/out": fmap(probe)})
    for c in "xyz":
        out[f"interp/values_{c}"] = vals[c]
    fmap._scaling = 2.5
    out["interp/out_scaled"] = fmap(probe)
    fmap._scaling = 1.0
    const = Field(dim=0, field={"x": 0.1, "y": -0.2, "z": 0.3}, scaling=2.0)
    out["interp/out_const"] = const(probe)
    out["interp/out_zero"] = Field.zero(3)(probe)
    out["interp/out_scaled_field"] = field.ScaledField(fmap, scale=3.0, offset=0.25)(probe)
    # CompositeField.__call__ fails above 100 points in the reference (its
    # Numba branch uses prange, which field.py never imports, field.py:644-648),
    # so composites are evaluated through its <= 100-point NumPy branch.
    def in_chunks(f, pts, size=100):
        return np.concatenate([f(pts[i:i + size]) for i in range(0, pts.shape[0], size)])

    out["interp/out_composite"] = in_chunks(field.CompositeField([fmap, const], [0.5, -1.5]), probe)
    out["interp/out_sub"] = in_chunks(fmap - const, probe)

    # -- tracking through a non-uniform, composite, scaled field --------------
    rng = np.random.default_rng(12)
    m = 64
    r0 = np.stack([rng.uniform(-0.03, 0.03, m), rng.uniform(-0.03, 0.05, m), rng.uniform(0.0, 0.05, m)], 1)
    v0 = np.stack([rng.normal(0, 2e5, m), rng.normal(0, 2e5, m), rng.uniform(5e5, 2e6, m)], 1)
    b_tot = field.CompositeField([fmap, const], [1e-2, 1.0])
    e_tot = 1e5 * fmap
    ion = species.IonSpecies("proton")
    for alg in ["boris", "rk4_rel", "vay_rel"]:
        rh, vh, _ = Pusher(ion, alg).track_batch(r0, v0, e_tot, b_tot, 300, 1e-10, 7)
        out[f"mixfield/{alg}/r_hist"] = rh
        out[f"mixfield/{alg}/v_hist"] = vh
    out.update({"mixfield/r0": r0, "mixfield/v0": v0})

    # -- rec_every not dividing nsteps; one particle; zero particles ----------
    p = Pusher(wl.species, "boris")
    rh, vh, _ = p.track_batch(wl.r0[:5], wl.v0[:5], ef, bf, 10, wl.dt, 3)
    out["edge/rec3/r_hist"], out["edge/rec3/v_hist"] = rh, vh
    rh, vh = p.track(wl.r0[7], wl.v0[7], ef, bf, 10, wl.dt, 4)
    out["edge/single/r_hist"], out["edge/single/v_hist"] = rh, vh
    rn, vn = p.push(wl.r0[7], wl.v0[7], ef, bf, wl.dt)
    out["edge/push/r"], out["edge/push/v"] = rn, vn
    rn, vn = p.push_batch(wl.r0[:9], wl.v0[:9], ef, bf, wl.dt)
    out["edge/push_batch/r"], out["edge/push_batch/v"] = rn, vn
    rh, vh, act = p.track_batch(np.zeros((0, 3)), np.zeros((0, 3)), ef, bf, 4, wl.dt, 2)
    out["edge/empty/r_hist_shape"] = np.array(rh.shape)
    pr = Pusher(wl.species, "rk4_rel")
    rh, vh = pr.track(wl.r0[7], wl.v0[7], ef, bf, 10, wl.dt, 5)
    out["edge/single_rk4_rel/r_hist"], out["edge/single_rk4_rel/v_hist"] = rh, vh

    # -- ParticleDistribution boundary conversion and moments -----------------
    # (particles.py:71-117, :393-457, :693-788)
    rfin = out["c1/boris/r_hist"][-1]
    vfin = out["c1/boris/v_hist"][-1]
    pd = particles.ParticleDistribution(species=wl.species, x_vec=rfin, p_vec=np.zeros_like(rfin))
    pd.set_p_from_v_vec(vfin)
    pd.recalculate_all()
    out["pd/p_vec"] = pd.p_vec
    out["pd/v_vec"] = pd.v_vec
    out["pd/centroid"] = pd.centroid
    out["pd/x_std"] = pd._x_std_vec
    out["pd/xp_std"] = pd._xp_std_vec
    out["pd/corr"] = np.array([pd._xxp_std, pd._yyp_std, pd._xyp_std, pd._yxp_std])
    out["pd/emittance"] = pd.get_emittances(normalized=False)
    out["pd/emittance_n"] = pd.get_emittances(normalized=True)
    out["pd/ekin"] = pd.ekin_mev
    out["pd/ekin_mean"] = np.float64(pd.mean_energy_mev)
    out["pd/ekin_std"] = np.float64(pd.rms_energy_spread_mev)
    out["pd/mass_mev"] = np.float64(wl.species.mass_mev)

    dest = HERE / "reference_golden.npz"
    np.savez_compressed(dest, **out)
    print("wrote", dest, dest.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
