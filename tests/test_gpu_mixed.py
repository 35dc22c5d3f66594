"""Mixed-precision form vs the float64 oracle.

Error metric (per particle, max over the bunch and all records):
|r - r_ref| / max(|r_ref|, half-width of the map) and |v - v_ref| / |v_ref|.
Target: <= 1e-6 relative position error for the fused Boris push on the RF
gap workload over its full 2e4 steps."""
import numpy as np
import pytest

from oracle import pusher_oracle as orc
from pypatools_b200 import PusherGPU, RFModulation, workloads
from tests.helpers import rel_pos_err, rel_vel_err, gpu_fields, half_width

pytestmark = pytest.mark.gpu


def _oracle_fields_sparse(wl):
    """Oracle maps with all-zero components dropped (same values, less memory)."""
    def clean(vals):
        if vals is None:
            return orc.ZeroField()
        return orc.MapField(wl.grid, {c: (None if vals[c] is None or not np.any(vals[c]) else vals[c])
                                      for c in "xyz"})
    return clean(wl.e_values), clean(wl.b_values)


def test_mixed_boris_rf_gap_full_length_vs_oracle(cuda):
    wl = workloads.rf_gap_protons(n=256, nsteps=20000, rec_every=500)
    e, b = gpu_fields(wl)
    rf = RFModulation(wl.rf_frequency, wl.rf_phase)
    rh, vh, _ = PusherGPU(wl.species, "boris", precision="mixed").track_batch(
        wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, wl.rec_every, rf=rf)
    oe, ob = _oracle_fields_sparse(wl)
    ro, vo, _ = orc.track_batch("boris", wl.species.q_over_m, wl.r0, wl.v0, oe, ob, wl.nsteps, wl.dt,
                                wl.rec_every, rf=(2 * np.pi * wl.rf_frequency, wl.rf_phase))
    err_r = rel_pos_err(rh, ro, half_width(wl))
    err_v = rel_vel_err(vh, vo)
    print(f"mixed boris rf gap: max rel pos err {err_r:.3e}, vel {err_v:.3e}")
    assert err_r <= 1e-6
    assert err_v <= 1e-6


def test_mixed_boris_matches_fp64_gpu_at_scale(cuda):
    # 65536 particles, full length: mixed vs the (oracle-pinned) float64 GPU path
    wl = workloads.rf_gap_protons(n=65536, nsteps=20000, rec_every=500)
    e, b = gpu_fields(wl)
    rf = RFModulation(wl.rf_frequency, wl.rf_phase)
    out = {}
    for prec in ("fp64", "mixed"):
        out[prec] = PusherGPU(wl.species, "boris", precision=prec, snapshot="device").track_batch(
            wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, wl.rec_every, rf=rf)
    rh = out["mixed"][0].cpu().numpy()
    ro = out["fp64"][0].cpu().numpy()
    err_r = rel_pos_err(rh, ro, half_width(wl))
    print(f"mixed vs fp64 (65536 x 2e4): max rel pos err {err_r:.3e}")
    assert err_r <= 1e-6


def test_mixed_boris_rf_gap_error_bar_at_scale(cuda):
    """The headline bar at scale: 1e6 protons of the RF-gap workload for its
    full 2e4 steps (41 records), the mixed form against the float64 form
    (pinned to the reference and the oracle at 1e-10): every particle within
    1e-6 relative position error at every record."""
    import torch
    from pypatools_b200.device_fields import DeviceFields
    from pypatools_b200.pusher import DeviceTracker
    dev = torch.device("cuda", 0)
    wl = workloads.rf_gap_protons(n=1_000_000)
    e, b = gpu_fields(wl)
    r0, v0 = torch.from_numpy(wl.r0).to(dev), torch.from_numpy(wl.v0).to(dev)
    ph = torch.from_numpy(wl.rf_phase).to(dev)
    hist = {}
    for prec in ("fp64", "mixed"):
        df = DeviceFields(e, b, prec, dev)
        tr = DeviceTracker("boris", wl.species.q_over_m, df, wl.n, wl.nsteps, wl.dt, wl.rec_every, prec,
                           rf_omega=2 * np.pi * wl.rf_frequency, rf_phase=ph, device=dev)
        tr.load(r0, v0)
        tr.run(wl.nsteps, 300, sort_every=300, long_chunk=1000)
        assert tr.device_status() == 0
        hist[prec] = tr.r_hist
        del tr, df
    num = torch.linalg.vector_norm(hist["mixed"] - hist["fp64"], dim=2)
    den = torch.clamp(torch.linalg.vector_norm(hist["fp64"], dim=2), min=half_width(wl))
    rel = (num / den).amax(dim=0)
    print(f"mixed vs fp64 (1e6 x 2e4): max {float(rel.max()):.3e}, p99 {float(torch.quantile(rel, 0.99)):.3e}, "
          f"over 1e-6: {int((rel > 1e-6).sum())}")
    assert bool(torch.isfinite(rel).all())
    assert float(rel.max()) <= 1e-6


def test_mixed_boris_quad_solenoid(cuda, golden):
    wl = workloads.quad_solenoid_protons()
    e, b = gpu_fields(wl)
    rh, vh, _ = PusherGPU(wl.species, "boris", precision="mixed").track_batch(wl.r0, wl.v0, e, b, 1000, wl.dt, 500)
    err_r = rel_pos_err(rh, golden["c1/boris/r_hist"], half_width(wl))
    err_v = rel_vel_err(vh, golden["c1/boris/v_hist"])
    print(f"mixed boris quad solenoid: pos {err_r:.3e} vel {err_v:.3e}")
    # float32 map values (the reference's are float64) bound this at ~1e-7
    assert err_r <= 1e-6 and err_v <= 1e-6


def _per_particle(r, r_ref, half):
    num = np.linalg.norm(r - r_ref, axis=2)
    den = np.maximum(np.linalg.norm(r_ref, axis=2), half)
    return (num / den).max(axis=0)


# Electrons rotate ~0.09 rad per step in this field with the reference's
# non-relativistic Boris, so the float32 rotation adds ~1e-8 relative error
# per step; once positions differ by ~1e-7 some particles leave the map one
# step apart, and the 1 MV/m field at the map face (fill 0 outside) turns that
# into a 1e-3-level velocity difference.  The bounds below are on the median
# and on the first record (before any exit); max and p90 are reported.
@pytest.mark.parametrize("alg,p50_bound,first_bound", [("boris", 1e-5, 1e-4), ("vay_rel", 1e-2, 5e-2),
                                                       ("rk4_rel", 5e-6, 5e-5)])
def test_mixed_electron_sweep_error_report(cuda, golden, alg, p50_bound, first_bound):
    wl = workloads.radial_e_solenoid_electrons(n=128)
    e, b = gpu_fields(wl)
    rh, vh, _ = PusherGPU(wl.species, alg, precision="mixed").track_batch(wl.r0, wl.v0, e, b, 10000, wl.dt, 2500)
    half = half_width(wl)
    per = _per_particle(rh, golden[f"c2/{alg}/r_hist"], half)
    first = rel_pos_err(rh[1], golden[f"c2/{alg}/r_hist"][1], half)
    err_v = rel_vel_err(vh, golden[f"c2/{alg}/v_hist"])
    print(f"mixed {alg} electrons: pos p50 {np.median(per):.3e} p90 {np.quantile(per, 0.9):.3e} "
          f"max {per.max():.3e}; first record {first:.3e}; vel max {err_v:.3e}")
    assert np.isfinite(per).all()
    assert np.median(per) <= p50_bound
    assert first <= first_bound


def test_mixed_rejects_unsupported(cuda):
    wl = workloads.quad_solenoid_protons(n=8)
    e, b = gpu_fields(wl)
    with pytest.raises(NotImplementedError):
        PusherGPU(wl.species, "yoshida", precision="mixed").track_batch(wl.r0, wl.v0, e, b, 2, wl.dt)


def _uniform_bz_workload(species, n, ke_mev, seed):
    """A bunch gyrating in a uniform Bz = 1 T map (33^3 nodes over +-5 cm):
    |u| is a constant of the motion."""
    from pypatools_b200.species import IonSpecies
    from pypatools_b200.constants import CLIGHT
    rng = np.random.default_rng(seed)
    ion = IonSpecies(species)
    g = np.linspace(-0.05, 0.05, 33)
    shape = (33, 33, 33)
    gamma = 1.0 + ke_mev / ion.mass_mev
    speed = np.sqrt(1.0 - 1.0 / gamma ** 2) * CLIGHT
    d = rng.normal(size=(n, 3))
    d[:, 2] *= 0.01
    d /= np.linalg.norm(d, axis=1)[:, None]
    r0 = rng.uniform(-2e-3, 2e-3, (n, 3))
    b = {"x": None, "y": None, "z": np.ones(shape)}
    return ion, (g, g.copy(), g.copy()), b, r0, d * speed


@pytest.mark.parametrize("alg", ["boris_rel", "vay"])
@pytest.mark.parametrize("species,ke,dt", [("proton", 0.01, 1e-10), ("electron", 1.0, 2e-13)])
def test_mixed_u_pushers_conserve_speed_in_pure_b(cuda, alg, species, ke, dt):
    """Relativistic Boris and Vay rotate u without changing |u| in a pure
    magnetic field; the mixed form accumulates float32 increments in a float
    pair, so |u| (and |v|) stays put to a few float32 roundings of the
    increments, far below 1e-6 over 3000 steps."""
    from pypatools_b200 import Field
    ion, grid, b, r0, v0 = _uniform_bz_workload(species, 512, ke, 7)
    g = {"x": grid[0], "y": grid[1], "z": grid[2]}
    bf = Field.from_arrays(g, b)
    rh, vh, _ = PusherGPU(ion, alg, precision="mixed").track_batch(r0, v0, Field.zero(3), bf, 3000, dt, 1000)
    speed = np.linalg.norm(vh, axis=2)
    drift = np.abs(speed[1:] / speed[0] - 1.0).max()
    inside = np.all(np.abs(rh) < 0.05, axis=(0, 2)).mean()
    print(f"mixed {alg} {species}: max relative |v| change {drift:.3e}, inside the map {inside:.2f}")
    assert inside > 0.99
    assert drift < 1e-6


@pytest.mark.parametrize("alg", ["boris_rel", "vay"])
def test_mixed_u_pushers_vs_oracle_electrons(cuda, alg):
    """The electron pusher sweep's bunch (C2: 10 keV - 10 MeV, radial 1 MV/m E,
    solenoid B) against the float64 oracle's boris_rel / vay: the error is
    reported; the median is bounded (the fast rotation and the fill-0 map
    faces amplify float32 effects, as for the mixed non-relativistic Boris)."""
    wl = workloads.radial_e_solenoid_electrons(n=128)
    e, b = gpu_fields(wl)
    rh, vh, _ = PusherGPU(wl.species, alg, precision="mixed").track_batch(wl.r0, wl.v0, e, b, 10000, wl.dt, 2500)
    oe, ob = _oracle_fields_sparse(wl)
    ro, vo, _ = orc.track_batch(alg, wl.species.q_over_m, wl.r0, wl.v0, oe, ob, 10000, wl.dt, 2500)
    per = _per_particle(rh, ro, half_width(wl))
    first = rel_pos_err(rh[1], ro[1], half_width(wl))
    print(f"mixed {alg} electrons vs oracle: pos p50 {np.median(per):.3e} p90 {np.quantile(per, 0.9):.3e} "
          f"max {per.max():.3e}; first record {first:.3e}")
    assert np.isfinite(per).all()
    assert np.median(per) <= 1e-4
    assert first <= 1e-3


@pytest.mark.parametrize("alg", ["boris_rel", "vay"])
def test_mixed_u_pushers_rf_gap_vs_fp64(cuda, alg):
    """1 MeV protons through the RF gap (65536, full 2e4 steps): the mixed
    relativistic pushers against their float64 form."""
    wl = workloads.rf_gap_protons(n=65536, nsteps=20000, rec_every=500)
    e, b = gpu_fields(wl)
    rf = RFModulation(wl.rf_frequency, wl.rf_phase)
    out = {}
    for prec in ("fp64", "mixed"):
        out[prec] = PusherGPU(wl.species, alg, precision=prec, snapshot="device").track_batch(
            wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, wl.rec_every, rf=rf)
    rh = out["mixed"][0].cpu().numpy()
    ro = out["fp64"][0].cpu().numpy()
    per = _per_particle(rh, ro, half_width(wl))
    print(f"mixed {alg} rf gap vs fp64 (65536 x 2e4): max {per.max():.3e}, p99 {np.quantile(per, 0.99):.3e}")
    assert per.max() <= 1e-6
