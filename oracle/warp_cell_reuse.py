"""How often a warp could skip its corner gather on the RF-gap map crossing
(ANALYSIS INFRASTRUCTURE ONLY: runs the oracle on the CPU; nothing in the
package imports it).

A proton of the RF-gap bunch (1 MeV, dt = 1e-11 s, 0.78 mm cells) stays in
its cell for ~5 steps, so a thread that kept its 8 corner records in
registers could skip the gather on most of its own steps.  A warp issues
the gather whenever ANY of its 32 lanes changed cell, so what matters is
the share of warp-steps in which no active lane did.  This script tracks
a bunch sample through the map with the oracle (every step recorded),
re-sorts it by cell every 300 steps as the bench's schedule does, groups 32
consecutive particles into a warp, and prints both shares.

    python -m oracle.warp_cell_reuse
"""
import numpy as np

from . import cpu_baseline as cb


def main(n=8192, steps=1300, sort_every=300):
    from pypatools_b200 import workloads
    wl = workloads.rf_gap_protons(n=n, nsteps=steps)
    omap, keep = cb.make_map(wl.grid, wl.e_values, wl.b_values)
    rh, _ = cb.track("boris", wl.r0, wl.v0, omap, steps, wl.dt, wl.species.q_over_m, rec=1,
                     omega=2 * np.pi * wl.rf_frequency, phase=wl.rf_phase)
    del keep
    lo = np.array([g[0] for g in wl.grid])
    h = np.array([g[1] - g[0] for g in wl.grid])
    nn = np.array([len(g) for g in wl.grid])
    cell = np.floor((rh - lo) / h).astype(np.int64)                  # (steps + 1, n, 3)
    inside = np.all((cell >= 0) & (cell < nn - 1), axis=2)
    key = (cell[..., 0] * nn[1] + cell[..., 1]) * nn[2] + cell[..., 2]
    changed = np.any(cell[1:] != cell[:-1], axis=2)                   # (steps, n)
    act = inside[1:] & inside[:-1]
    same_thread = 1.0 - changed[act].mean()
    skip, total = 0, 0
    for s0 in range(0, steps, sort_every):
        order = np.argsort(np.where(inside[s0], key[s0], np.iinfo(np.int64).max), kind="stable")
        for s in range(s0, min(s0 + sort_every, steps)):
            ch = changed[s][order].reshape(-1, 32)
            a = act[s][order].reshape(-1, 32)
            live = a.any(axis=1)
            total += int(live.sum())
            skip += int((live & ~(ch & a).any(axis=1)).sum())
    print(f"in-map particle-steps in the same cell as the step before: {same_thread:.3f}")
    print(f"in-map warp-steps in which no active lane changed cell: {skip / total:.4f} of {total}")
    return same_thread, skip / total


if __name__ == "__main__":
    main()
