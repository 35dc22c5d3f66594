"""Seeded synthetic field-map files in the reference's loader formats.

``write_cases(directory)`` writes the same files every time; the fixture
generator (make_golden_loaders.py) reads them with the reference's loaders and
the tests read them with this package's.  Returns {case: (path, kwargs)}."""
import os

import numpy as np


def _fmt(a):
    return " ".join(repr(float(v)) for v in np.ravel(a))


def write_cases(directory):
    rng = np.random.default_rng(31)
    os.makedirs(directory, exist_ok=True)
    cases = {}

    # OPERA: 3D magnetic in cm / Gauss, rows with z fastest
    nx, ny, nz = 5, 4, 3
    gx, gy, gz = np.linspace(-2.0, 2.0, nx), np.linspace(-1.5, 1.5, ny), np.linspace(0.0, 4.0, nz)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    b = rng.normal(0, 500.0, (3, nx, ny, nz))
    path = os.path.join(directory, "opera3d.table")
    with open(path, "w") as fh:
        fh.write(f"{nx} {ny} {nz} 2\n1 X [CM]\n2 Y [CM]\n3 Z [CM]\n4 BX [GAUSS]\n5 BY [GAUSS]\n6 BZ [GAUSS]\n0\n")
        for row in zip(X.ravel(), Y.ravel(), Z.ravel(), b[0].ravel(), b[1].ravel(), b[2].ravel()):
            fh.write(_fmt(row) + "\n")
    cases["opera3d"] = (path, {})

    # OPERA: 2D (x, y) in mm, Bz in Tesla
    nx, ny = 6, 3
    X, Y = np.meshgrid(np.linspace(0.0, 50.0, nx), np.linspace(-10.0, 10.0, ny), indexing="ij")
    path = os.path.join(directory, "opera2d.table")
    with open(path, "w") as fh:
        fh.write(f"{nx} {ny} 1\n1 X [mm]\n2 Y [mm]\n3 BZ [Tesla]\n0\n")
        for row in zip(X.ravel(), Y.ravel(), rng.uniform(0.5, 1.5, nx * ny)):
            fh.write(_fmt(row) + "\n")
    cases["opera2d"] = (path, {})

    # OPERA: electric 3D in m / V/cm, Ey missing
    nx, ny, nz = 3, 3, 4
    X, Y, Z = np.meshgrid(np.linspace(0, 0.1, nx), np.linspace(0, 0.2, ny), np.linspace(-0.1, 0.1, nz),
                          indexing="ij")
    path = os.path.join(directory, "opera_e.table")
    with open(path, "w") as fh:
        fh.write(f"{nx} {ny} {nz}\n1 X [m]\n2 Y [m]\n3 Z [m]\n4 EX [V/cm]\n5 EZ [V/cm]\n0\n")
        for row in zip(X.ravel(), Y.ravel(), Z.ravel(), rng.normal(0, 1e3, X.size), rng.normal(0, 1e3, X.size)):
            fh.write(_fmt(row) + "\n")
    cases["opera_e"] = (path, {})

    # OPERA: field columns only, positions from extents (cm)
    nx, ny, nz = 4, 3, 2
    path = os.path.join(directory, "opera_ext.table")
    with open(path, "w") as fh:
        fh.write(f"{nx} {ny} {nz}\n1 BX [Tesla]\n2 BY [Tesla]\n3 BZ [Tesla]\n0\n")
        for row in rng.normal(0, 0.1, (nx * ny * nz, 3)):
            fh.write(_fmt(row) + "\n")
    cases["opera_ext"] = (path, {"extents": [(-3.0, 3.0), (-2.0, 2.0), (0.0, 5.0)],
                                 "extents_dims": ["X", "Y", "Z"]})

    # COMSOL: 3D magnetic in cm, rows shuffled
    nx, ny, nz = 4, 3, 5
    X, Y, Z = np.meshgrid(np.linspace(-1, 1, nx), np.linspace(0, 2, ny), np.linspace(-2, 2, nz), indexing="ij")
    rows = np.column_stack([X.ravel(), Y.ravel(), Z.ravel(), rng.normal(0, 0.2, (X.size, 3))])
    rows = rows[rng.permutation(rows.shape[0])]
    path = os.path.join(directory, "comsol3d.comsol")
    with open(path, "w") as fh:
        fh.write("% Model: synthetic\n% Version: COMSOL 5.6\n% Date: none\n% Dimension: 3\n"
                 f"% Nodes: {X.size}\n% Expressions: 3\n% Description: Magnetic flux density\n"
                 "% Length unit: cm\n% x y z mf.Bx (T) mf.By (T) mf.Bz (T)\n")
        for row in rows:
            fh.write(_fmt(row) + "\n")
    cases["comsol3d"] = (path, {})

    # COMSOL: 2D electric (x, z) in mm, V/m, labels with prefixes and digits
    nx, nz = 5, 4
    X, Z = np.meshgrid(np.linspace(0, 40, nx), np.linspace(-30, 30, nz), indexing="ij")
    rows = np.column_stack([X.ravel(), Z.ravel(), rng.normal(0, 5e4, (X.size, 2))])
    rows = rows[rng.permutation(rows.shape[0])]
    path = os.path.join(directory, "comsol2d.comsol")
    with open(path, "w") as fh:
        fh.write("% Model: synthetic\n% Version: COMSOL 5.6\n% Date: none\n% Dimension: 2\n"
                 f"% Nodes: {X.size}\n% Expressions: 2\n% Description: Electric field\n"
                 "% Length unit: mm\n% x z es.Ex2 (V/m) mires.Ez (V/m)\n")
        for row in rows:
            fh.write(_fmt(row) + "\n")
    cases["comsol2d"] = (path, {})

    # OPAL midplane: r 10..200 mm, theta 0..357.5 deg, Bz in kG
    nr, nth = 20, 144
    r = np.linspace(10.0, 200.0, nr)[:, None]
    th = np.deg2rad(np.linspace(0.0, 357.5, nth))[None, :]
    bz = 10.0 * (1.0 + 0.2 * np.cos(4 * th) * (r / 200.0)) + rng.normal(0, 0.01, (nr, nth))
    path = os.path.join(directory, "midplane.dat")
    with open(path, "w") as fh:
        fh.write("10.0\n10.0\n0.0\n2.5\n" f"{nth}\n{nr}\n")
        for row in bz:
            fh.write(_fmt(row) + "\n")
    cases["opal"] = (path, {})
    cases["opal_cut"] = (path, {"r_cutoff": 0.15, "nx": 61, "ny": 41})
    cases["opal_cyl"] = (path, {"cartesian_grid": False})

    # AIMA AGORA: three z slices (0, 10, 20 mm) of br, bf, bz; cm and degrees
    adir = os.path.join(directory, "aima")
    os.makedirs(adir, exist_ok=True)
    nth, nr = 36, 12
    r = np.linspace(0.0, 12 * 2.0, nr, endpoint=False)[:, None]
    th = np.deg2rad(np.linspace(0.0, 36 * 10.0, nth, endpoint=False))[None, :]
    for zmm in (0, 10, 20):
        comps = {"br": 0.01 * (r / 24.0) * np.sin(4 * th) * (1 + zmm / 50.0),
                 "bf": 0.02 * np.cos(3 * th) * (r / 24.0) ** 2 + 0 * zmm,
                 "bz": 1.0 + 0.1 * np.cos(4 * th) * (r / 24.0) - 0.001 * zmm}
        for comp, vals in comps.items():
            vals = vals + rng.normal(0, 1e-4, (nr, nth))
            with open(os.path.join(adir, f"fieldZ{zmm:03d}-{comp}.map"), "w") as fh:
                fh.write("synthetic slice\n" f"{nth} {nr}\n0.0 2.0\n0.0 10.0\n")
                for row in vals:
                    fh.write(_fmt(row) + "\n")
                fh.write("end\n")
    cases["aima"] = (adir, {"interp_resolution": 81})
    cases["aima_mirror"] = (adir, {"mirror": True, "interp_resolution": 51})
    return cases
