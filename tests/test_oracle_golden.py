"""Pin the CPU oracle to the reference: every case below was produced by
running the reference's own code (tests/golden/make_golden.py); the oracle
restatement must reproduce it.  Tolerances: the reference runs Numba with
fastmath (contraction/reassociation), the oracle plain NumPy, so agreement is
to rounding, far inside the 1e-10 parity budget of the GPU path."""
import numpy as np
import pytest

from oracle import pusher_oracle as orc
from pypatools_b200 import workloads
from pypatools_b200.species import IonSpecies, PRESETS
from tests.helpers import rel_pos_err, rel_vel_err, oracle_fields, half_width

TOL = 1e-11


def test_species_q_over_m_bit_identical(golden):
    for name in PRESETS:
        assert IonSpecies(name).q_over_m == golden[f"species/{name}/q_over_m"]


def test_workload_inputs_match_fixture(golden):
    wl = workloads.quad_solenoid_protons()
    np.testing.assert_array_equal(wl.r0, golden["c1/r0"])
    np.testing.assert_array_equal(wl.v0, golden["c1/v0"])
    wl2 = workloads.radial_e_solenoid_electrons(n=128)
    np.testing.assert_array_equal(wl2.r0, golden["c2/r0"])
    np.testing.assert_array_equal(wl2.v0, golden["c2/v0"])


def test_oracle_boris_quad_solenoid_full(golden):
    wl = workloads.quad_solenoid_protons()
    e, b = oracle_fields(wl)
    rh, vh, act = orc.track_batch("boris", wl.species.q_over_m, wl.r0, wl.v0, e, b, 1000, wl.dt, 500)
    assert rh.shape == golden["c1/boris/r_hist"].shape
    assert rel_pos_err(rh, golden["c1/boris/r_hist"], half_width(wl)) < TOL
    assert rel_vel_err(vh, golden["c1/boris/v_hist"]) < TOL
    assert act.all() and golden["c1/boris/active"].all()


@pytest.mark.parametrize("alg", ["leapfrog", "rk4", "yoshida", "vay_rel", "rk4_rel", "yoshida_rel"])
def test_oracle_other_algorithms_quad_solenoid(golden, alg):
    wl = workloads.quad_solenoid_protons()
    sub = slice(0, 4096, 16)
    e, b = oracle_fields(wl)
    rh, vh, _ = orc.track_batch(alg, wl.species.q_over_m, wl.r0[sub], wl.v0[sub], e, b, 1000, wl.dt, 250)
    assert rel_pos_err(rh, golden[f"c1/{alg}/r_hist"], half_width(wl)) < TOL
    assert rel_vel_err(vh, golden[f"c1/{alg}/v_hist"]) < TOL


@pytest.mark.parametrize("alg", ["boris", "vay_rel", "rk4_rel"])
def test_oracle_radial_e_solenoid_electrons(golden, alg):
    wl = workloads.radial_e_solenoid_electrons(n=128)
    e, b = oracle_fields(wl)
    rh, vh, _ = orc.track_batch(alg, wl.species.q_over_m, wl.r0, wl.v0, e, b, 10000, wl.dt, 2500)
    # 1e4 steps of relativistic electrons; the reference 'vay_rel' runs |v| up
    # to its 0.9999 c clamp and amplifies rounding to ~2e-11: the 1e-10 bar.
    assert rel_pos_err(rh, golden[f"c2/{alg}/r_hist"], half_width(wl)) < 1e-10
    assert rel_vel_err(vh, golden[f"c2/{alg}/v_hist"]) < 1e-10


def _interp_case(golden):
    grid = (golden["interp/gx"], golden["interp/gy"], golden["interp/gz"])
    vals = {c: golden[f"interp/values_{c}"] for c in "xyz"}
    return grid, vals, golden["interp/probe"]


def test_oracle_interpolation_edges(golden):
    grid, vals, probe = _interp_case(golden)
    fmap = orc.MapField(grid, vals)
    np.testing.assert_allclose(fmap(probe), golden["interp/out"], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(orc.MapField(grid, vals, scaling=2.5)(probe), golden["interp/out_scaled"],
                               rtol=1e-14, atol=1e-14)
    const = orc.ConstField([0.1, -0.2, 0.3], scaling=2.0)
    np.testing.assert_array_equal(const(probe), golden["interp/out_const"])
    np.testing.assert_array_equal(orc.ZeroField()(probe), golden["interp/out_zero"])
    np.testing.assert_allclose(orc.ScaledOracleField(fmap, 3.0, 0.25)(probe), golden["interp/out_scaled_field"],
                               rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(orc.CompositeOracleField([fmap, const], [0.5, -1.5])(probe),
                               golden["interp/out_composite"], rtol=1e-14, atol=1e-14)
    np.testing.assert_allclose(orc.CompositeOracleField([fmap, const], [1.0, -1.0])(probe),
                               golden["interp/out_sub"], rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("alg", ["boris", "rk4_rel", "vay_rel"])
def test_oracle_nonuniform_composite_tracking(golden, alg):
    grid, vals, _ = _interp_case(golden)
    fmap = orc.MapField(grid, vals)
    const = orc.ConstField([0.1, -0.2, 0.3], scaling=2.0)
    b = orc.CompositeOracleField([fmap, const], [1e-2, 1.0])
    e = orc.ScaledOracleField(fmap, 1e5, 0.0)
    qm = IonSpecies("proton").q_over_m
    rh, vh, _ = orc.track_batch(alg, qm, golden["mixfield/r0"], golden["mixfield/v0"], e, b, 300, 1e-10, 7)
    assert rel_pos_err(rh, golden[f"mixfield/{alg}/r_hist"], 0.05) < TOL
    assert rel_vel_err(vh, golden[f"mixfield/{alg}/v_hist"]) < TOL


def test_oracle_track_edge_cases(golden):
    wl = workloads.quad_solenoid_protons()
    e, b = oracle_fields(wl)
    qm = wl.species.q_over_m
    rh, vh, _ = orc.track_batch("boris", qm, wl.r0[:5], wl.v0[:5], e, b, 10, wl.dt, 3)
    np.testing.assert_allclose(rh, golden["edge/rec3/r_hist"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(vh, golden["edge/rec3/v_hist"], rtol=1e-13, atol=0)
    rs, vs = orc.track_single("boris", qm, wl.r0[7], wl.v0[7], e, b, 10, wl.dt, 4)
    np.testing.assert_allclose(rs, golden["edge/single/r_hist"], rtol=1e-13)
    np.testing.assert_allclose(vs, golden["edge/single/v_hist"], rtol=1e-13)
    rs, vs = orc.track_single("rk4_rel", qm, wl.r0[7], wl.v0[7], e, b, 10, wl.dt, 5)
    np.testing.assert_allclose(rs, golden["edge/single_rk4_rel/r_hist"], rtol=1e-13)
    np.testing.assert_allclose(vs, golden["edge/single_rk4_rel/v_hist"], rtol=1e-13)
    rn, vn = orc.push_step("boris", wl.r0[:9], wl.v0[:9], orc._Fields(e, b), 0.0, wl.dt, qm)
    np.testing.assert_allclose(rn, golden["edge/push_batch/r"], rtol=1e-14)
    np.testing.assert_allclose(vn, golden["edge/push_batch/v"], rtol=1e-14)
    rh, _, _ = orc.track_batch("boris", qm, np.zeros((0, 3)), np.zeros((0, 3)), e, b, 4, wl.dt, 2)
    np.testing.assert_array_equal(rh.shape, golden["edge/empty/r_hist_shape"])


def test_oracle_bunch_moments(golden):
    x = golden["c1/boris/r_hist"][-1]
    v = golden["c1/boris/v_hist"][-1]
    p = orc.momenta_from_velocities(v)
    np.testing.assert_allclose(p, golden["pd/p_vec"], rtol=1e-15)
    np.testing.assert_allclose(orc.velocities_from_momenta(p), golden["pd/v_vec"], rtol=1e-15)
    m = orc.bunch_moments(x, p, float(golden["pd/mass_mev"]))
    np.testing.assert_allclose(m["centroid"], golden["pd/centroid"], rtol=1e-12)
    np.testing.assert_allclose(m["x_std"], golden["pd/x_std"], rtol=1e-12)
    np.testing.assert_allclose(m["xp_std"], golden["pd/xp_std"], rtol=1e-12)
    np.testing.assert_allclose([m["xxp"], m["yyp"], m["xyp"], m["yxp"]], golden["pd/corr"], rtol=1e-10)
    np.testing.assert_allclose(m["emittance"], golden["pd/emittance"], rtol=1e-9)
    np.testing.assert_allclose(m["emittance_n"], golden["pd/emittance_n"], rtol=1e-9)
    np.testing.assert_allclose(orc.kinetic_energies(p, float(golden["pd/mass_mev"])), golden["pd/ekin"],
                               rtol=1e-12)
    np.testing.assert_allclose(m["ekin_mean"], golden["pd/ekin_mean"], rtol=1e-12)
    np.testing.assert_allclose(m["ekin_std"], golden["pd/ekin_std"], rtol=1e-9)


DT_GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "dt_golden.npz"


@pytest.fixture(scope="module")
def dt_golden():
    with np.load(DT_GOLDEN) as d:
        return {k: d[k] for k in d.files}


def _dt_workload(tag):
    if tag == "quad":
        return workloads.quad_solenoid_protons(n=96, nsteps=400, seed=21)
    return workloads.radial_e_solenoid_electrons(n=64, nsteps=800, seed=22)


@pytest.mark.parametrize("tag", ["quad", "radial"])
@pytest.mark.parametrize("alg", ["rk4", "rk4_rel"])
def test_oracle_rk4_per_particle_dt(dt_golden, tag, alg):
    """The reference's batch RK4 step with one dt per particle
    (pusher.py:815-816), through track_batch and push_batch."""
    wl = _dt_workload(tag)
    np.testing.assert_array_equal(wl.r0, dt_golden[f"{tag}/r0"])
    e, b = oracle_fields(wl)
    dt = dt_golden[f"{tag}/dt"]
    steps, rec = int(dt_golden[f"{tag}/nsteps"]), int(dt_golden[f"{tag}/rec"])
    rh, vh, _ = orc.track_batch(alg, wl.species.q_over_m, wl.r0, wl.v0, e, b, steps, dt, rec)
    assert rel_pos_err(rh, dt_golden[f"{tag}/{alg}/r_hist"], half_width(wl)) < TOL
    assert rel_vel_err(vh, dt_golden[f"{tag}/{alg}/v_hist"]) < TOL
    rn, vn = orc.push_step(alg, wl.r0, wl.v0, orc._Fields(e, b), 0.0, dt, wl.species.q_over_m)
    np.testing.assert_allclose(rn, dt_golden[f"{tag}/{alg}/push_r"], rtol=1e-14)
    np.testing.assert_allclose(vn, dt_golden[f"{tag}/{alg}/push_v"], rtol=1e-14)


def test_particle_distribution_boundary_conversions(golden):
    """The package's own ParticleDistribution (not the oracle's copy): the
    reference's per-component v -> beta*gamma -> v conversions
    (particles.py:71-117, :393-457) on the C1 final state."""
    from pypatools_b200 import ParticleDistribution
    x = golden["c1/boris/r_hist"][-1]
    v = golden["c1/boris/v_hist"][-1]
    pd = ParticleDistribution(species=IonSpecies("proton"), x_vec=x, p_vec=np.zeros_like(x), recalculate=False)
    pd.set_p_from_v_vec(v)
    np.testing.assert_allclose(pd.p_vec, golden["pd/p_vec"], rtol=1e-15, atol=0)
    np.testing.assert_allclose(pd.v_vec, golden["pd/v_vec"], rtol=1e-15, atol=0)
    np.testing.assert_array_equal(pd.x_vec, x)
