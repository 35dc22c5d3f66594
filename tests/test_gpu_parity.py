"""Plain (float64) GPU path vs the reference: golden trajectories produced by
the reference itself (tests/golden), and the CPU oracle where the reference
has no counterpart (RF time dependence, boris_rel, vay).  Bar: <= 1e-10
relative position and velocity error after the stated step counts."""
import numpy as np
import pytest

from oracle import pusher_oracle as orc
from pypatools_b200 import PusherGPU, Field, ScaledField, CompositeField, RFModulation, workloads
from pypatools_b200.moments import bunch_moments
from pypatools_b200.species import IonSpecies
from tests.helpers import rel_pos_err, rel_vel_err, gpu_fields, oracle_fields, half_width

pytestmark = pytest.mark.gpu
TOL = 1e-10


def test_boris_quad_solenoid_full(cuda, golden):
    wl = workloads.quad_solenoid_protons()
    e, b = gpu_fields(wl)
    rh, vh, act = PusherGPU(wl.species, "boris").track_batch(wl.r0, wl.v0, e, b, 1000, wl.dt, 500)
    ref_r, ref_v = golden["c1/boris/r_hist"], golden["c1/boris/v_hist"]
    assert rh.shape == ref_r.shape and vh.shape == ref_v.shape
    assert rel_pos_err(rh, ref_r, half_width(wl)) < TOL
    assert rel_vel_err(vh, ref_v) < TOL
    assert act.dtype == bool and act.all()


@pytest.mark.parametrize("alg", ["leapfrog", "rk4", "yoshida", "vay_rel", "rk4_rel", "yoshida_rel"])
def test_other_algorithms_quad_solenoid(cuda, golden, alg):
    wl = workloads.quad_solenoid_protons()
    sub = slice(0, 4096, 16)
    e, b = gpu_fields(wl)
    rh, vh, _ = PusherGPU(wl.species, alg).track_batch(wl.r0[sub], wl.v0[sub], e, b, 1000, wl.dt, 250)
    assert rel_pos_err(rh, golden[f"c1/{alg}/r_hist"], half_width(wl)) < TOL
    assert rel_vel_err(vh, golden[f"c1/{alg}/v_hist"]) < TOL


@pytest.mark.parametrize("alg", ["boris", "vay_rel", "rk4_rel"])
def test_radial_e_solenoid_electrons(cuda, golden, alg):
    wl = workloads.radial_e_solenoid_electrons(n=128)
    e, b = gpu_fields(wl)
    rh, vh, _ = PusherGPU(wl.species, alg).track_batch(wl.r0, wl.v0, e, b, 10000, wl.dt, 2500)
    assert rel_pos_err(rh, golden[f"c2/{alg}/r_hist"], half_width(wl)) < TOL
    assert rel_vel_err(vh, golden[f"c2/{alg}/v_hist"]) < TOL


def _interp_fields(golden):
    g = {"x": golden["interp/gx"], "y": golden["interp/gy"], "z": golden["interp/gz"]}
    vals = {c: golden[f"interp/values_{c}"] for c in "xyz"}
    return Field.from_arrays(g, vals), Field(dim=0, field={"x": 0.1, "y": -0.2, "z": 0.3}, scaling=2.0)


def test_field_evaluation_edges(cuda, golden):
    fmap, const = _interp_fields(golden)
    probe = golden["interp/probe"]
    kw = dict(rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(fmap(probe), golden["interp/out"], **kw)
    fmap.scaling = 2.5
    np.testing.assert_allclose(fmap(probe), golden["interp/out_scaled"], **kw)
    fmap.scaling = 1.0
    np.testing.assert_array_equal(const(probe), golden["interp/out_const"])
    np.testing.assert_array_equal(Field.zero(3)(probe), golden["interp/out_zero"])
    np.testing.assert_allclose(ScaledField(fmap, 3.0, 0.25)(probe), golden["interp/out_scaled_field"], **kw)
    np.testing.assert_allclose(CompositeField([fmap, const], [0.5, -1.5])(probe), golden["interp/out_composite"], **kw)
    np.testing.assert_allclose((fmap - const)(probe), golden["interp/out_sub"], **kw)


@pytest.mark.parametrize("alg", ["boris", "rk4_rel", "vay_rel"])
def test_nonuniform_composite_tracking(cuda, golden, alg):
    fmap, const = _interp_fields(golden)
    b = CompositeField([fmap, const], [1e-2, 1.0])
    e = 1e5 * fmap
    rh, vh, _ = PusherGPU(IonSpecies("proton"), alg).track_batch(golden["mixfield/r0"], golden["mixfield/v0"],
                                                               e, b, 300, 1e-10, 7)
    assert rel_pos_err(rh, golden[f"mixfield/{alg}/r_hist"], 0.05) < TOL
    assert rel_vel_err(vh, golden[f"mixfield/{alg}/v_hist"]) < TOL


def test_edge_cases(cuda, golden):
    wl = workloads.quad_solenoid_protons()
    e, b = gpu_fields(wl)
    p = PusherGPU(wl.species, "boris")
    rh, vh, _ = p.track_batch(wl.r0[:5], wl.v0[:5], e, b, 10, wl.dt, 3)
    np.testing.assert_allclose(rh, golden["edge/rec3/r_hist"], rtol=1e-12)
    np.testing.assert_allclose(vh, golden["edge/rec3/v_hist"], rtol=1e-12)
    rs, vs = p.track(wl.r0[7], wl.v0[7], e, b, 10, wl.dt, 4)
    np.testing.assert_allclose(rs, golden["edge/single/r_hist"], rtol=1e-12)
    np.testing.assert_allclose(vs, golden["edge/single/v_hist"], rtol=1e-12)
    rn, vn = p.push(wl.r0[7], wl.v0[7], e, b, wl.dt)
    np.testing.assert_allclose(rn, golden["edge/push/r"], rtol=1e-13)
    np.testing.assert_allclose(vn, golden["edge/push/v"], rtol=1e-13)
    rn, vn = p.push_batch(wl.r0[:9], wl.v0[:9], e, b, wl.dt)
    np.testing.assert_allclose(rn, golden["edge/push_batch/r"], rtol=1e-13)
    np.testing.assert_allclose(vn, golden["edge/push_batch/v"], rtol=1e-13)
    rh, vh, act = p.track_batch(np.zeros((0, 3)), np.zeros((0, 3)), e, b, 4, wl.dt, 2)
    np.testing.assert_array_equal(rh.shape, golden["edge/empty/r_hist_shape"])
    assert act.shape == (0,)
    rs, vs = PusherGPU(wl.species, "rk4_rel").track(wl.r0[7], wl.v0[7], e, b, 10, wl.dt, 5)
    np.testing.assert_allclose(rs, golden["edge/single_rk4_rel/r_hist"], rtol=1e-12)
    np.testing.assert_allclose(vs, golden["edge/single_rk4_rel/v_hist"], rtol=1e-12)
    # zero steps: records 0 only; Boris half step back then forward
    rh, vh, _ = p.track_batch(wl.r0[:3], wl.v0[:3], e, b, 0, wl.dt, 1)
    ro, vo, _ = orc.track_batch("boris", wl.species.q_over_m, wl.r0[:3], wl.v0[:3], *oracle_fields(wl), 0, wl.dt, 1)
    np.testing.assert_allclose(rh, ro, rtol=1e-14)
    np.testing.assert_allclose(vh, vo, rtol=1e-13)


def test_bunch_moments_vs_reference(cuda, golden):
    x = golden["c1/boris/r_hist"][-1]
    v = golden["c1/boris/v_hist"][-1]
    m = bunch_moments(x, v, float(golden["pd/mass_mev"]))
    np.testing.assert_allclose(m["centroid"], golden["pd/centroid"], rtol=1e-12)
    np.testing.assert_allclose(m["x_std"], golden["pd/x_std"], rtol=1e-12)
    np.testing.assert_allclose(m["xp_std"], golden["pd/xp_std"], rtol=1e-12)
    np.testing.assert_allclose([m["xxp"], m["yyp"], m["xyp"], m["yxp"]], golden["pd/corr"], rtol=1e-10)
    np.testing.assert_allclose(m["emittance"], golden["pd/emittance"], rtol=1e-9)
    np.testing.assert_allclose(m["emittance_n"], golden["pd/emittance_n"], rtol=1e-9)
    np.testing.assert_allclose(m["ekin_mean"], golden["pd/ekin_mean"], rtol=1e-12)
    np.testing.assert_allclose(m["ekin_std"], golden["pd/ekin_std"], rtol=1e-9)


@pytest.mark.parametrize("alg", ["boris", "vay_rel", "rk4_rel", "rk4"])
def test_rf_time_dependent_vs_oracle(cuda, alg):
    wl = workloads.rf_gap_protons(n=128, nsteps=3000, nodes=129, rec_every=500)
    e, b = gpu_fields(wl)
    rf = RFModulation(wl.rf_frequency, wl.rf_phase)
    rh, vh, _ = PusherGPU(wl.species, alg).track_batch(wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, wl.rec_every, rf=rf)
    oe, ob = oracle_fields(wl)
    ro, vo, _ = orc.track_batch(alg, wl.species.q_over_m, wl.r0, wl.v0, oe, ob, wl.nsteps, wl.dt, wl.rec_every,
                                rf=(2 * np.pi * wl.rf_frequency, wl.rf_phase))
    assert rel_pos_err(rh, ro, half_width(wl)) < TOL
    assert rel_vel_err(vh, vo) < TOL


@pytest.mark.parametrize("alg", ["boris_rel", "vay"])
def test_u_state_algorithms_vs_oracle(cuda, alg):
    wl = workloads.radial_e_solenoid_electrons(n=64, nsteps=2000)
    e, b = gpu_fields(wl)
    rh, vh, _ = PusherGPU(wl.species, alg).track_batch(wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, 500)
    oe, ob = oracle_fields(wl)
    ro, vo, _ = orc.track_batch(alg, wl.species.q_over_m, wl.r0, wl.v0, oe, ob, wl.nsteps, wl.dt, 500)
    assert rel_pos_err(rh, ro, half_width(wl)) < TOL
    assert rel_vel_err(vh, vo) < TOL


@pytest.mark.parametrize("tag", ["quad", "radial"])
@pytest.mark.parametrize("alg", ["rk4", "rk4_rel"])
def test_rk4_per_particle_dt(cuda, tag, alg):
    """One dt per particle, as the reference's batch RK4 step takes it
    (pusher.py:815-816): track_batch and push_batch against the reference's
    own outputs (tests/golden/dt_golden.npz), cell-sorted or not."""
    from pathlib import Path
    with np.load(Path(__file__).resolve().parent / "golden" / "dt_golden.npz") as d:
        gold = {k: d[k] for k in d.files}
    if tag == "quad":
        wl = workloads.quad_solenoid_protons(n=96, nsteps=400, seed=21)
    else:
        wl = workloads.radial_e_solenoid_electrons(n=64, nsteps=800, seed=22)
    e, b = gpu_fields(wl)
    dt = gold[f"{tag}/dt"]
    steps, rec = int(gold[f"{tag}/nsteps"]), int(gold[f"{tag}/rec"])
    for sort_every in (0, 50):
        p = PusherGPU(wl.species, alg, sort_every=sort_every, steps_per_launch=70)
        rh, vh, _ = p.track_batch(wl.r0, wl.v0, e, b, steps, dt, rec)
        assert rel_pos_err(rh, gold[f"{tag}/{alg}/r_hist"], half_width(wl)) < TOL
        assert rel_vel_err(vh, gold[f"{tag}/{alg}/v_hist"]) < TOL
    rn, vn = PusherGPU(wl.species, alg).push_batch(wl.r0, wl.v0, e, b, dt)
    np.testing.assert_allclose(rn, gold[f"{tag}/{alg}/push_r"], rtol=1e-13, atol=0)
    np.testing.assert_allclose(vn, gold[f"{tag}/{alg}/push_v"], rtol=1e-13, atol=0)


def test_sector_ring_fp64_vs_c_oracle(cuda):
    """The large-scale configuration's map, 512^3 float32 Bz over a 1 m cube
    (the one-component record layout, float64 on the device, 1.1 GB): 1000
    protons of its bunch for 2000 steps (about three turns), the float64 form
    against the C oracle at 1e-10; the mixed form's error is reported."""
    from oracle import cpu_baseline
    wl = workloads.sector_ring_protons(n=1000, nsteps=2000, rec_every=500)
    e, b = gpu_fields(wl)
    omap, keep = cpu_baseline.make_map(wl.grid, wl.e_values, wl.b_values)
    ro, vo = cpu_baseline.track("boris", wl.r0, wl.v0, omap, wl.nsteps, wl.dt, wl.species.q_over_m, wl.rec_every)
    del keep
    rh, vh, _ = PusherGPU(wl.species, "boris").track_batch(wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, wl.rec_every)
    assert rel_pos_err(rh, ro, half_width(wl)) < TOL
    assert rel_vel_err(vh, vo) < TOL
    rm, vm, _ = PusherGPU(wl.species, "boris", precision="mixed").track_batch(wl.r0, wl.v0, e, b, wl.nsteps,
                                                                               wl.dt, wl.rec_every)
    print(f"sector ring 1000 x 2000, mixed vs C oracle: pos {rel_pos_err(rm, ro, half_width(wl)):.3e} "
          f"vel {rel_vel_err(vm, vo):.3e}")
    assert rel_pos_err(rm, ro, half_width(wl)) < 1e-5
