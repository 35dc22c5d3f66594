"""Field-map file loaders with the reference's return format.

Restates the loaders of src/PyPATools/field_src/field_loaders.py behind the
same names, arguments and result dictionaries (``grid``, ``values``, ``dim``,
``field_type``, ``metadata``; lengths in m, B in T, E in V/m):

* ``load_opera_table``   OPERA ``.table``              (field_loaders.py:65-256)
* ``load_comsol``        COMSOL ``.comsol`` export     (:259-486)
* ``load_opal_midplane`` OPAL CARBONCYCL midplane      (:489-670)
* ``load_aima_agora``    AIMA AGORA ``*Z<z>-<c>.map``  (:673-928)
* ``load_h5part``        H5Part (needs h5py)           (:931-1050)

and ``Field.from_file``'s dispatch by extension (field.py:284-343).  Text is
parsed on the host; the cylindrical maps' resampling onto a Cartesian grid
(the reference runs scipy's RegularGridInterpolator on the CPU) runs on the
GPU (``ppt_polar_to_cartesian``).

Kept from the reference: its unit tables, grid detection, C-order reshapes
(an OPERA or COMSOL file is read as [x][y][z] with z fastest, whatever order
its rows are in), zero components for missing ones, the AIMA reader's skipped
last line of each file and its r grid (``linspace(r0, nr dr, nr,
endpoint=False)``), and its error types.  Not kept: blank lines break the
reference's OPERA and OPAL readers (its own tests of them fail on the trailing
whitespace line of their inputs); here blank lines are skipped.  Progress
prints are left out.
"""
import gc
import os
import re
import warnings

import numpy as np

from . import _lib

UNIT_CONVERSIONS = {
    "length": {"mm": 0.001, "cm": 0.01, "m": 1.0},
    "magnetic": {"gauss": 1e-4, "kgauss": 0.1, "tesla": 1.0, "t": 1.0},
    "electric": {"v/mm": 1000.0, "v/cm": 100.0, "v/m": 1.0},
}


def _numbers(lines):
    """All whitespace-separated numbers of ``lines`` as one float64 array
    (parsed in C, without a Python object per number: a 256^3 map has 1e8)."""
    text = " ".join(lines)
    if not text.strip():
        return np.zeros(0)
    with warnings.catch_warnings():
        # numpy warns (and stops) at text it cannot read: make that an error
        warnings.simplefilter("error")
        try:
            return np.fromstring(text, dtype=np.float64, sep=" ")
        except (DeprecationWarning, ValueError) as exc:
            raise ValueError(f"could not convert the map's values to numbers: {exc}")


def _unit_kind(unit):
    u = unit.lower()
    for kind in ("length", "magnetic", "electric"):
        if u in UNIT_CONVERSIONS[kind]:
            return kind
    return None


# ---------------------------------------------------------------------------
# OPERA .table
# ---------------------------------------------------------------------------

def load_opera_table(filename, extents=None, extents_dims=None):
    """OPERA .table map: a line of node counts, ``<col> <label> [<unit>]``
    column lines up to a line ``0``, then one row per node."""
    if not os.path.exists(filename):
        raise FileNotFoundError(f"File not found: {filename}")
    if extents is not None and extents_dims is None:
        raise ValueError("extents_dims must be specified when using extents")
    try:
        with open(filename, "r") as fh:
            counts = np.array([int(tok) - 1 for tok in fh.readline().split()])[:3]
            columns = {}
            n_len = n_b = n_e = 0
            last_col = -1
            for line in fh:
                line = line.strip()
                if line == "0":
                    break
                parts = line.split()
                last_col = int(parts[0]) - 1
                found = re.search(r"\[(.*?)]", line)
                if not found:
                    raise ValueError(f"No unit found for column {parts[1]}")
                columns[parts[1]] = {"column": last_col, "unit": found.group(1)}
                kind = _unit_kind(found.group(1))
                n_len += kind == "length"
                n_b += kind == "magnetic"
                n_e += kind == "electric"
            if extents is not None:
                for k, label in enumerate(extents_dims):
                    columns[label] = {"column": last_col + k + 1, "unit": "cm"}
                    n_len += 1
            # node counts by axis: counts[0] is x's when the file has x, else
            # y's, else z's; an axis the file lacks has one node
            if "X" in columns:
                n = {"X": counts[0] + 1, "Y": counts[1] + 1 if "Y" in columns else 1,
                     "Z": counts[2] + 1 if "Z" in columns else 1}
            elif "Y" in columns:
                n = {"X": 1, "Y": counts[0] + 1, "Z": counts[1] + 1 if "Z" in columns else 1}
            elif "Z" in columns:
                n = {"X": 1, "Y": 1, "Z": counts[0] + 1}
            else:
                raise KeyError("X")
            dim = int(np.count_nonzero(counts > 0))
            if n_e > 0 and n_b > 0:
                raise ValueError("Mixed E and B fields not supported")
            field_type = "electric" if n_e > 0 else "magnetic"
            rows = n["X"] * n["Y"] * n["Z"]
            n_cols = n_len + n_e + n_b
            table = np.zeros((rows, n_cols))
            body = _numbers(fh.readlines())
            if extents is not None:
                gx, gy, gz = (np.linspace(lim[0], lim[1], n[a]) for lim, a in zip(extents, "XYZ"))
                mx, my, mz = np.meshgrid(gx, gy, gz, indexing="ij")
                table[:, -3], table[:, -2], table[:, -1] = mx.ravel(), my.ravel(), mz.ravel()
                width = n_cols - n_len
                if body.size != rows * width:
                    raise ValueError(f"expected {rows} rows of {width} values")
                table[:, :width] = body.reshape(rows, width)
            else:
                if body.size != rows * n_cols:
                    raise ValueError(f"expected {rows} rows of {n_cols} values")
                table[:] = body.reshape(rows, n_cols)
    except Exception as exc:
        raise RuntimeError(f"Error reading OPERA table file: {exc}")
    grid = {}
    for a in "XYZ":
        if a in columns and _unit_kind(columns[a]["unit"]) == "length":
            grid[a.lower()] = np.unique(table[:, columns[a]["column"]]) * \
                UNIT_CONVERSIONS["length"][columns[a]["unit"].lower()]
    kind = "magnetic" if field_type == "magnetic" else "electric"
    prefix = "B" if field_type == "magnetic" else "E"
    shape = [n["X"], n["Y"], n["Z"]]
    values = {}
    for c in "XYZ":
        label = prefix + c
        if label in columns:
            scale = UNIT_CONVERSIONS[kind].get(columns[label]["unit"].lower(), 1.0)
            values[c.lower()] = table[:, columns[label]["column"]].reshape(shape) * scale
        else:
            values[c.lower()] = np.zeros(shape)
    del table
    gc.collect()
    return {"grid": grid, "values": values, "dim": dim, "field_type": field_type,
            "metadata": {"n_points": n, "units_original": {k: v["unit"] for k, v in columns.items()},
                         "filename": os.path.basename(filename)}}


# ---------------------------------------------------------------------------
# COMSOL export
# ---------------------------------------------------------------------------

_COMSOL_LABELS = {
    "x": "X", "y": "Y", "z": "Z", "r": "R", "phi": "PHI", "theta": "THETA",
    "mf.Bx": "BX", "mf.By": "BY", "mf.Bz": "BZ", "Bx": "BX", "By": "BY", "Bz": "BZ",
    "mf.Br": "BR", "mf.Bphi": "BPHI", "mf.Btheta": "BTHETA",
    "es.Ex": "EX", "es.Ey": "EY", "es.Ez": "EZ", "es.Er": "ER", "es.Ephi": "EPHI", "es.Etheta": "ETHETA",
}
_COMSOL_SPATIAL = ("X", "Y", "Z", "R", "PHI", "THETA")
_COMSOL_OUT = {"BX": "x", "BY": "y", "BZ": "z", "BR": "r", "BPHI": "phi", "BTHETA": "theta",
               "EX": "x", "EY": "y", "EZ": "z", "ER": "r", "EPHI": "phi", "ETHETA": "theta"}


def load_comsol(filename):
    """COMSOL export: a 9-line ``%`` header (dimension, node count, length
    unit, column labels with units) and one row per node in any order."""
    if not os.path.exists(filename):
        raise FileNotFoundError(f"File not found: {filename}")
    try:
        with open(filename, "r") as fh:
            header = [fh.readline().strip() for _ in range(9)]
        int(header[3].split()[2])           # "% Dimension: n" (checked, not used)
        array_len = int(header[4].split()[2])
        l_unit = header[7].split()[3]
        line = header[8]
        b_unit = e_unit = None
        if "(T)" in line:
            b_unit, field_type = "T", "magnetic"
        elif "(V/cm)" in line:
            e_unit, field_type = "V/cm", "electric"
        elif "(V/m)" in line:
            e_unit, field_type = "V/m", "electric"
        elif "mf.B" in line:
            b_unit, field_type = "T", "magnetic"
        elif "es.E" in line:
            e_unit, field_type = "V/m", "electric"
        else:
            raise ValueError("Cannot determine field type from header")
        tokens = line.split()
        labels = tokens[:4] + re.split(r"\([a-zA-Z/]+\)", "".join(tokens[4:]))
        columns, spatial, fields = {}, [], []
        col = 0
        for label in labels:
            if label in ("%", "(T)", "(V/cm)", "(V/m)", "", " "):
                continue
            name = _COMSOL_LABELS.get(re.sub(r"side|mir|sec|cpl|\d+", "", label))
            if name is None:
                continue          # an unknown label takes no column number
            columns[name] = {"column": col}
            if name in _COMSOL_SPATIAL:
                columns[name]["unit"] = l_unit
                spatial.append(name)
            elif name.startswith("B") and b_unit:
                columns[name]["unit"] = b_unit
                fields.append(name)
            elif name.startswith("E") and e_unit:
                columns[name]["unit"] = e_unit
                fields.append(name)
            col += 1
        if not spatial:
            raise ValueError("No spatial coordinates found in file")
        if not fields:
            raise ValueError("No field components found in file")
        dim = len(spatial)
        table = np.loadtxt(filename, skiprows=9, max_rows=array_len)
        if table.ndim == 1:
            table = table.reshape(1, -1)
    except Exception as exc:
        raise RuntimeError(f"Error reading COMSOL file: {exc}")
    # rows ordered with the first coordinate slowest, the last fastest
    keys = [table[:, columns[c]["column"]] for c in reversed(spatial)]
    order = np.argsort(keys[0]) if dim == 1 else np.lexsort(keys)
    table = table[order]
    n, grid = {}, {}
    l_scale = UNIT_CONVERSIONS["length"].get(l_unit.lower(), 1.0)
    for c in spatial:
        nodes = np.unique(table[:, columns[c]["column"]])
        n[c] = len(nodes)
        grid[c.lower()] = nodes * l_scale
    if np.prod(list(n.values())) != array_len:
        raise ValueError(f"Grid size mismatch: {np.prod(list(n.values()))} expected vs {array_len} in file")
    shape = [n[c] for c in spatial]
    kind = "magnetic" if field_type == "magnetic" else "electric"
    values = {}
    for name in fields:
        scale = UNIT_CONVERSIONS[kind].get(columns[name]["unit"].lower(), 1.0)
        values[_COMSOL_OUT.get(name, name.lower())] = table[:, columns[name]["column"]].reshape(shape) * scale
    for c in "xyz":
        values.setdefault(c, np.zeros(shape))
        grid.setdefault(c, np.array([0.0]))
    del table
    gc.collect()
    return {"grid": grid, "values": values, "dim": dim, "field_type": field_type,
            "metadata": {"n_points": n, "spatial_dims": spatial, "field_dims": fields,
                         "units_original": {k: v["unit"] for k, v in columns.items() if "unit" in v},
                         "filename": os.path.basename(filename)}}


# ---------------------------------------------------------------------------
# cylindrical maps -> Cartesian grid (GPU)
# ---------------------------------------------------------------------------

def polar_to_cartesian(r_nodes, theta_nodes, comps, x, y, r_scale=1.0, want=(True, True, True)):
    """Resample (B_r, B_theta, B_z) given on the (r, theta [deg]) node grid
    (``comps``: three (nr, nt) arrays or None) onto the Cartesian nodes x, y
    at one z.  Returns [B_x, B_y, B_z] as (nx, ny) float64 arrays (None where
    ``want`` is False).  Runs ``ppt_polar_to_cartesian``."""
    import torch
    r_nodes, theta_nodes, x, y = (np.asarray(a, dtype=np.float64) for a in (r_nodes, theta_nodes, x, y))
    if any(a.ndim != 1 for a in (r_nodes, theta_nodes, x, y)):
        raise ValueError("r_nodes, theta_nodes, x and y must be 1D")
    if len(comps) != 3 or len(want) != 3:
        raise ValueError("comps and want hold the (r, theta, z) components: three entries each")
    for c in comps:
        if c is not None and np.shape(c) != (r_nodes.shape[0], theta_nodes.shape[0]):
            raise ValueError(f"a component of shape {np.shape(c)} on a ({r_nodes.shape[0]}, "
                             f"{theta_nodes.shape[0]}) (r, theta) node grid")
    if not torch.cuda.is_available():
        raise RuntimeError("the cylindrical-map resampling runs on the GPU (no CPU fallback)")
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device())

    def up(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)

    d_r, d_t, d_x, d_y = up(r_nodes), up(theta_nodes), up(x), up(y)
    d_c = [None if c is None else up(c) for c in comps]
    nx, ny = d_x.shape[0], d_y.shape[0]
    d_o = [torch.empty((nx, ny), dtype=torch.float64, device=dev) if w else None for w in want]
    g = _lib.PolarGrid(d_r.shape[0], d_t.shape[0], d_r.data_ptr(), d_t.data_ptr())
    cp = (_lib.c_void_p * 3)(*[None if c is None else c.data_ptr() for c in d_c])
    op = (_lib.c_void_p * 3)(*[None if o is None else o.data_ptr() for o in d_o])
    _lib.check(lib.ppt_polar_to_cartesian(g, cp, nx, d_x.data_ptr(), ny, d_y.data_ptr(), float(r_scale), op,
                                          _lib.stream_handle()))
    return [None if o is None else o.cpu().numpy() for o in d_o]


# ---------------------------------------------------------------------------
# OPAL CARBONCYCL midplane
# ---------------------------------------------------------------------------

def load_opal_midplane(filename, r_cutoff=None, scaling=1.0, cartesian_grid=True, nx=None, ny=None):
    """OPAL midplane Bz: r0, dr [mm], theta0, dtheta [deg], n_theta, n_r, then
    Bz [kG] with theta fastest; resampled onto an x-y grid unless
    ``cartesian_grid`` is False."""
    if not os.path.exists(filename):
        raise FileNotFoundError(f"File not found: {filename}")
    if os.path.splitext(filename)[1] != ".dat":
        raise ValueError("File extension must be '.dat'")
    try:
        with open(filename, "r") as fh:
            sr, dr, sth, dth = (float(fh.readline().strip()) for _ in range(4))
            nth = int(fh.readline().strip())
            nr = int(fh.readline().strip())
            rest = fh.readlines()
    except Exception as exc:
        raise RuntimeError(f"Error reading OPAL midplane file: {exc}")
    bz = scaling * 0.1 * _numbers(rest)     # kG -> T
    r_nodes = np.linspace(sr, sr + (nr - 1) * dr, nr)          # mm
    th_nodes = np.linspace(sth, sth + (nth - 1) * dth, nth)    # deg
    bz_cyl = bz.reshape(nr, nth)
    if r_cutoff is not None:
        bz_cyl[r_nodes > r_cutoff * 1000.0, :] = 0.0
    meta = {"r_range": (sr, sr + (nr - 1) * dr), "theta_range": (sth, sth + (nth - 1) * dth),
            "n_points": {"r": nr, "theta": nth}}
    if not cartesian_grid:
        meta.update({"r_cutoff": r_cutoff, "scaling": scaling, "filename": os.path.basename(filename)})
        return {"grid": {"r": r_nodes * 0.001, "theta": th_nodes, "z": np.array([0.0])},
                "values": {"r": np.zeros_like(bz_cyl), "theta": np.zeros_like(bz_cyl), "z": bz_cyl},
                "dim": 2, "field_type": "magnetic", "coordinate_system": "cylindrical", "metadata": meta}
    r_max = r_nodes[-1] * 0.001
    if r_cutoff is not None:
        r_max = min(r_max, r_cutoff)
    if nx is None:
        nx = int(2 * r_max / (dr * 0.001)) + 1
    if ny is None:
        ny = nx
    x = np.linspace(-r_max, r_max, nx)
    y = np.linspace(-r_max, r_max, ny)
    _, _, bz_cart = polar_to_cartesian(r_nodes, th_nodes, (None, None, bz_cyl), x, y, r_scale=1000.0,
                                       want=(False, False, True))
    if r_cutoff is not None:
        gx, gy = np.meshgrid(x, y, indexing="ij")
        bz_cart[np.sqrt(gx ** 2 + gy ** 2) > r_cutoff] = 0.0
    meta.update({"n_cartesian": {"x": nx, "y": ny}, "r_cutoff": r_cutoff, "scaling": scaling,
                 "filename": os.path.basename(filename)})
    return {"grid": {"x": x, "y": y, "z": np.array([0.0])},
            "values": {"x": np.zeros_like(bz_cart), "y": np.zeros_like(bz_cart), "z": bz_cart},
            "dim": 2, "field_type": "magnetic", "coordinate_system": "cartesian", "metadata": meta}


# ---------------------------------------------------------------------------
# AIMA AGORA slices
# ---------------------------------------------------------------------------

def load_aima_agora(path, mirror=False, interp_resolution=1000):
    """AIMA AGORA map: files ``*Z<z [mm]>-<br|bf|bz>.map`` of one directory,
    each a comment line, ``n_theta n_r``, ``r0 dr`` [cm], ``theta0 dtheta``
    [deg] and the values with theta fastest; every z slice resampled onto an
    ``interp_resolution``-square x-y grid, optionally mirrored about z = 0."""
    if os.path.isfile(path):
        directory = os.path.dirname(path)
    elif os.path.isdir(path):
        directory = path
    else:
        raise FileNotFoundError(f"Path not found: {path}")
    try:
        names = [e.name for e in os.scandir(directory) if e.is_file() and e.name.endswith(".map")]
    except OSError as exc:
        raise RuntimeError(f"Error scanning directory: {exc}") from exc
    if not names:
        raise FileNotFoundError(f"No .map files found in {directory}")
    files = []   # (path, component, z [mm])
    for name in names:
        try:
            z_text, rest = name.split("Z")[1].split("-")
            comp = rest.split(".")[0].lower()
            if comp not in ("br", "bf", "bz"):
                continue
            files.append((os.path.join(directory, name), comp, float(z_text)))
        except (IndexError, ValueError):   # not named <...>Z<z>-<component>.map
            continue
    if not files:
        raise ValueError("No valid .map files found")
    zsets = [{z for _, c, z in files if c == comp} for comp in ("br", "bf", "bz")]
    if not (zsets[0] == zsets[1] == zsets[2]):
        raise ValueError("Not all components have the same z positions. Maybe a file is missing?")

    def grid_params(fn):
        with open(fn, "r") as fh:
            fh.readline()
            nth_, nr_ = (int(v) for v in fh.readline().split())
            sr_, dr_ = (float(v) for v in fh.readline().split())
            sth_, dth_ = (float(v) for v in fh.readline().split())
        return nth_, nr_, sr_, dr_, sth_, dth_

    try:
        params = grid_params(files[0][0])
    except Exception as exc:
        raise RuntimeError(f"Error reading grid parameters from {files[0][0]}: {exc}")
    for fn, _, _ in files[1:]:
        if grid_params(fn) != params:
            raise ValueError(f"Grid mismatch in file {fn}")
    nth, nr, sr, dr, sth, dth = params
    r_nodes = np.linspace(sr, nr * dr, nr, endpoint=False)       # cm
    th_nodes = np.linspace(sth, nth * dth, nth, endpoint=False)  # deg
    z_unique = np.sort(np.unique([z for _, _, z in files])) / 10.0   # mm -> cm
    r_max = r_nodes[-1]
    x = np.linspace(-r_max, r_max, interp_resolution)
    y = np.linspace(-r_max, r_max, interp_resolution)
    if mirror:
        z_cart = np.concatenate((-z_unique[:0:-1], z_unique))
        offset = len(z_unique) - 1
    else:
        z_cart = z_unique
        offset = 0
    shape = (interp_resolution, interp_resolution, len(z_cart))
    bx, by, bz = np.zeros(shape), np.zeros(shape), np.zeros(shape)
    for j, z in enumerate(z_unique):
        comps = {}
        for comp in ("br", "bf", "bz"):
            match = [fn for fn, c, zz in files if c == comp and zz == 10.0 * z]
            if not match:
                raise ValueError(f"Missing {comp} component at z={10.0 * z} mm")
            with open(match[0], "r") as fh:
                lines = fh.readlines()[4:-1]     # the last line of each file is not read
            comps[comp] = _numbers(lines).reshape(nr, nth)
        i = j + offset
        bx[:, :, i], by[:, :, i], bz[:, :, i] = polar_to_cartesian(
            r_nodes, th_nodes, (comps["br"], comps["bf"], comps["bz"]), x, y)
        if mirror and j != 0:
            k = offset - j
            bx[:, :, k], by[:, :, k], bz[:, :, k] = -bx[:, :, i], -by[:, :, i], bz[:, :, i]
    return {"grid": {"x": x * 0.01, "y": y * 0.01, "z": z_cart * 0.01},
            "values": {"x": bx, "y": by, "z": bz}, "dim": 3, "field_type": "magnetic",
            "metadata": {"z_positions": z_unique, "n_files": len(names), "mirrored": mirror,
                         "interp_resolution": interp_resolution, "r_range": (sr, nr * dr),
                         "theta_range": (sth, nth * dth), "filename": os.path.basename(directory)}}


# ---------------------------------------------------------------------------
# H5Part
# ---------------------------------------------------------------------------

def load_h5part(filename):
    """H5Part map: the H field of ``Step#0/Block/Hfield`` (components ``0``,
    ``1``, ``2`` stored [z][y][x], attributes ``__Spacing__`` and
    ``__Origin__``), returned [x][y][z]."""
    if not os.path.exists(filename):
        raise FileNotFoundError(f"File not found: {filename}")
    try:
        import h5py
    except ImportError as exc:
        raise ImportError("load_h5part needs the h5py package") from exc
    h5 = None
    try:
        h5 = h5py.File(filename, "r")
        block = h5["Step#0"]["Block"]
        has_e = "Efield" in block
        if "Hfield" not in block:
            raise ValueError("No Hfield found in H5Part file")
        grp = block["Hfield"]
        comps = [np.array(grp[k]) for k in ("0", "1", "2")]
        spacing = grp.attrs["__Spacing__"]
        origin = grp.attrs["__Origin__"]
        nz, ny, nx = comps[0].shape
        axes = [origin[a] + np.arange(m) * spacing[a] for a, m in enumerate((nx, ny, nz))]
        values = [np.transpose(c, (2, 1, 0)) for c in comps]
        h5.close()
    except Exception as exc:
        if h5 is not None:
            h5.close()
        raise RuntimeError(f"Error reading H5Part file: {exc}")
    return {"grid": {"x": axes[0], "y": axes[1], "z": axes[2]},
            "values": {"x": values[0], "y": values[1], "z": values[2]}, "dim": 3, "field_type": "magnetic",
            "metadata": {"spacing": spacing, "origin": origin, "shape": (nx, ny, nz), "has_efield": has_e,
                         "filename": os.path.basename(filename)}}


LOADERS = {".h5": load_h5part, ".h5part": load_h5part, ".table": load_opera_table, ".comsol": load_comsol,
           ".dat": load_opal_midplane, ".map": load_aima_agora}
