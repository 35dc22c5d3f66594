"""Generate the 1D / 2D field fixture (fields12_golden.npz) by running the reference.

The reference's ``Field`` has 1D fields that vary along z and 2D fields that
vary along x and y (``_get_field_1d`` / ``_get_field_2d``,
src/PyPATools/field.py:457-489, over ``_interp1d_batch`` / ``_interp2d_batch``,
field_src/interpolators.py:192-257).  This script evaluates such fields and
tracks particles through them with the reference's own ``Pusher.track_batch``.

1D fields use the reference's 'scipy' interpolator backend: with the default
Numba backend, ``_get_field_1d`` hands the interpolator a 1-D array of M z
values, which ``NumbaInterpolator.__call__`` (interpolators.py:357-364) reads
as ONE point of dimension M and rejects for M > 1 ("Points have dimension M,
expected 1").  The fixture records that failure too.

    PYPATOOLS_REFERENCE_SRC=<checkout>/src python tests/golden/make_golden_fields12.py
"""
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from make_golden import load_reference  # noqa: E402


def sector_bz(gx, gy):
    """A four-sector cyclotron-like median-plane field in T."""
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    th = np.arctan2(Y, X)
    rr = np.hypot(X, Y)
    return 1.0 + 0.15 * np.cos(4.0 * th) * np.tanh(rr / 0.05) + 0.05 * rr


def probe_points(rng, lo, hi, nodes):
    pts = np.stack([rng.uniform(lo[0], hi[0], 600), rng.uniform(lo[1], hi[1], 600),
                    rng.uniform(lo[2], hi[2], 600)], axis=1)
    return np.concatenate([pts, nodes])


def main():
    pusher, field, species, particles = load_reference()
    Pusher, Field = pusher.Pusher, field.Field
    ion = species.IonSpecies("proton")
    out = {}
    rng = np.random.default_rng(21)

    # -- 2D field on a non-uniform (x, y) grid: evaluation -------------------
    gx = np.linspace(-0.3, 0.3, 61)
    gy = np.sort(np.concatenate([[-0.3, 0.3], rng.uniform(-0.3, 0.3, 39)]))
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    vals = {"x": 0.02 * Y, "y": 0.03 * X * Y, "z": sector_bz(gx, gy)}
    f2 = Field.from_arrays({"x": gx, "y": gy, "z": np.array([0.0])}, vals)
    assert f2.dim == 2
    nodes = np.array([[gx[0], gy[0], 0.0], [gx[-1], gy[-1], 5.0], [gx[7], gy[11], -1e3],
                      [np.nextafter(gx[-1], 1), 0.0, 0.0], [0.0, np.nextafter(gy[0], -1), 0.0],
                      [0.01, 0.02, 1e6]])
    probe = probe_points(rng, (-0.35, -0.35, -2.0), (0.35, 0.35, 2.0), nodes)
    out.update({"f2/gx": gx, "f2/gy": gy, "f2/probe": probe, "f2/out": f2(probe)})
    for c in "xyz":
        out[f"f2/values_{c}"] = vals[c]

    # -- 1D field along z: evaluation -----------------------------------------
    gz = np.sort(np.concatenate([[-0.2, 0.2], rng.uniform(-0.2, 0.2, 59)]))
    v1 = {"x": np.zeros_like(gz), "y": np.zeros_like(gz), "z": 2e6 * np.cos(np.pi * gz / 0.4)}
    try:
        Field.from_arrays({"z": gz}, v1)(np.zeros((4, 3)))
        out["f1/numba_batch_raises"] = np.int64(0)
    except ValueError as exc:
        out["f1/numba_batch_raises"] = np.int64(1)
        print("numba-backed 1D field, 4 points:", exc)
    f1 = Field.from_arrays({"z": gz}, v1, interpolator_backend="scipy")
    assert f1.dim == 1
    nodes = np.array([[0.0, 0.0, gz[0]], [3.0, -4.0, gz[-1]], [0.0, 0.0, gz[17]],
                      [0.0, 0.0, np.nextafter(gz[-1], 1)], [1e3, 1e3, 0.05]])
    probe = probe_points(rng, (-1.0, -1.0, -0.25), (1.0, 1.0, 0.25), nodes)
    out.update({"f1/gz": gz, "f1/probe": probe, "f1/out": f1(probe)})
    for c in "xyz":
        out[f"f1/values_{c}"] = v1[c]

    # -- tracking: protons on a ring through a uniform-grid 2D sector field --
    gxu = np.linspace(-0.3, 0.3, 121)
    gyu = np.linspace(-0.3, 0.3, 121)
    bz = sector_bz(gxu, gyu)
    zero = np.zeros_like(bz)
    b2 = Field.from_arrays({"x": gxu, "y": gyu}, {"x": zero, "y": zero, "z": bz})
    m = 128
    ekin = 1.0 * (1.0 + 0.01 * rng.uniform(-1, 1, m))            # MeV
    gamma = 1.0 + ekin / ion.mass_mev
    speed = 299792458.0 * np.sqrt(1.0 - 1.0 / gamma ** 2)
    r0 = np.stack([-0.1445 + rng.normal(0, 2e-3, m), rng.normal(0, 2e-3, m), rng.normal(0, 5e-3, m)], 1)
    ang = rng.normal(0, 3e-3, (m, 2))
    d = np.stack([ang[:, 0], np.ones(m), ang[:, 1]], 1)
    v0 = speed[:, None] * d / np.linalg.norm(d, axis=1, keepdims=True)
    out.update({"ring2d/gx": gxu, "ring2d/gy": gyu, "ring2d/bz": bz, "ring2d/r0": r0, "ring2d/v0": v0})
    for alg in ["boris", "vay_rel", "rk4_rel"]:
        rh, vh, _ = Pusher(ion, alg).track_batch(r0, v0, Field.zero(3), b2, 2000, 1e-10, 500)
        out[f"ring2d/{alg}/r_hist"] = rh
        out[f"ring2d/{alg}/v_hist"] = vh
        print("ring2d", alg, "done")

    # -- tracking: a 1D Ez(z) gap with a 1D solenoid Bz(z), both along z -----
    gzu = np.linspace(-0.2, 0.2, 201)
    ez = 3e6 * np.exp(-(gzu / 0.03) ** 2)
    bzs = 0.5 / (1.0 + (gzu / 0.08) ** 2)
    z1 = np.zeros_like(gzu)
    e1 = Field.from_arrays({"z": gzu}, {"x": z1, "y": z1, "z": ez}, interpolator_backend="scipy")
    b1 = Field.from_arrays({"z": gzu}, {"x": z1, "y": z1, "z": bzs}, interpolator_backend="scipy")
    m = 64
    r0 = np.stack([rng.normal(0, 1e-3, m), rng.normal(0, 1e-3, m), -0.19 + rng.uniform(0, 0.01, m)], 1)
    v0 = np.stack([rng.normal(0, 1e5, m), rng.normal(0, 1e5, m), rng.uniform(1.2e7, 1.4e7, m)], 1)
    out.update({"gap1d/gz": gzu, "gap1d/ez": ez, "gap1d/bz": bzs, "gap1d/r0": r0, "gap1d/v0": v0})
    for alg in ["boris", "rk4_rel"]:
        rh, vh, _ = Pusher(ion, alg).track_batch(r0, v0, e1, b1, 3000, 1e-11, 750)
        out[f"gap1d/{alg}/r_hist"] = rh
        out[f"gap1d/{alg}/v_hist"] = vh
        print("gap1d", alg, "done")

    dest = HERE / "fields12_golden.npz"
    np.savez_compressed(dest, **out)
    print("wrote", dest, dest.stat().st_size, "bytes")


if __name__ == "__main__":
    main()
