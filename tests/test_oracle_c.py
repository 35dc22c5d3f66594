"""The C oracle (the timed CPU baseline) against the reference's golden
trajectories and the NumPy oracle."""
import numpy as np
import pytest

from oracle import cpu_baseline, pusher_oracle as orc
from pypatools_b200 import workloads
from tests.helpers import rel_pos_err, rel_vel_err, half_width


@pytest.mark.parametrize("alg", ["boris", "vay_rel", "rk4_rel", "rk4", "leapfrog"])
def test_c_oracle_vs_reference_golden(golden, alg):
    wl = workloads.quad_solenoid_protons()
    omap, keep = cpu_baseline.make_map(wl.grid, wl.e_values, wl.b_values)
    if alg == "boris":
        r0, v0, rec, key = wl.r0, wl.v0, 500, "c1/boris"
    else:
        sub = slice(0, 4096, 16)
        r0, v0, rec, key = wl.r0[sub], wl.v0[sub], 250, f"c1/{alg}"
    rh, vh = cpu_baseline.track(alg, r0, v0, omap, 1000, wl.dt, wl.species.q_over_m, rec)
    assert rel_pos_err(rh, golden[f"{key}/r_hist"], half_width(wl)) < 1e-11
    assert rel_vel_err(vh, golden[f"{key}/v_hist"]) < 1e-11


def test_c_oracle_rf_vs_numpy_oracle():
    wl = workloads.rf_gap_protons(n=200, nsteps=600, nodes=65, rec_every=200)
    omap, keep = cpu_baseline.make_map(wl.grid, wl.e_values, wl.b_values)
    omega = 2 * np.pi * wl.rf_frequency
    rh, vh = cpu_baseline.track("boris", wl.r0, wl.v0, omap, wl.nsteps, wl.dt, wl.species.q_over_m, 200,
                                omega=omega, phase=wl.rf_phase)
    e = orc.MapField(wl.grid, wl.e_values)
    b = orc.MapField(wl.grid, wl.b_values)
    ro, vo, _ = orc.track_batch("boris", wl.species.q_over_m, wl.r0, wl.v0, e, b, wl.nsteps, wl.dt, 200,
                                rf=(omega, wl.rf_phase))
    assert rel_pos_err(rh, ro, half_width(wl)) < 1e-12
    assert rel_vel_err(vh, vo) < 1e-12
