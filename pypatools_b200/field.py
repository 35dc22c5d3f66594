"""Field objects with the reference's API, evaluated on the GPU.

Mirrors ``Field``, ``ScaledField``, ``CompositeField``, ``FieldMap`` and
``get_interpolator`` of the reference (src/PyPATools/field.py:101-755,
field_src/interpolators.py:533-610) for the pieces on the pusher path:
0D (constant) fields and 1D, 2D and 3D node-map fields, field algebra, and
point evaluation.  Evaluation goes through ``ppt_field_eval`` (one cell
lookup per point for all components) instead of three per-component Numba
passes.  As in the reference, a 1D field varies along z and a 2D field along
x and y (field.py:457-489).

The pusher accepts these objects and the reference's own equally (see
``device_fields``).  ``Field.from_file`` reads the reference's map formats
(``loaders``).
"""
import os
import pickle

import numpy as np

from . import _lib
from .device_fields import FieldCache

UNIT_SCALES = {"m": 1.0, "cm": 0.01, "mm": 0.001, "Tesla": 1.0, "T": 1.0, "Gauss": 1e-4,
               "kGauss": 0.1, "V/m": 1.0, "V/cm": 100.0, "V/mm": 1000.0}

_eval_cache = FieldCache(capacity=8)


def _evaluate(field, pts):
    """(M,3) float64 field values of ``field`` at ``pts`` on the GPU."""
    import torch
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
    if pts.ndim != 2 or pts.shape[1] != 3:
        raise ValueError(f"Points must have shape (M, 3), got {pts.shape}")
    m = pts.shape[0]
    if m == 0:
        return np.zeros((0, 3))
    df = _eval_cache.get(field, None, "fp64")
    lib = _lib.load()
    d_pts = torch.from_numpy(np.ascontiguousarray(pts)).to(df.device)
    d_out = torch.empty((m, 3), dtype=torch.float64, device=df.device)
    with torch.cuda.device(df.device):
        _lib.check(lib.ppt_field_eval(df.fields, m, d_pts.data_ptr(), d_out.data_ptr(), None,
                                      _lib.stream_handle()))
    return d_out.cpu().numpy()


class FieldBase:
    """Field protocol: ``field(pts (M,3)) -> (M,3)`` (field.py:68-98)."""

    def __call__(self, pts):
        raise NotImplementedError

    def gradient(self, pts):
        raise NotImplementedError("Gradient not implemented for this field type")

    def __add__(self, other):
        if isinstance(other, (int, float)):
            return ScaledField(self, offset=other)
        return CompositeField([self, other], [1.0, 1.0])

    def __sub__(self, other):
        if isinstance(other, (int, float)):
            return ScaledField(self, offset=-other)
        return CompositeField([self, other], [1.0, -1.0])

    def __mul__(self, scalar):
        return ScaledField(self, scale=scalar)

    def __rmul__(self, scalar):
        return self.__mul__(scalar)


class Field(FieldBase):
    """0D constant or 1D / 2D / 3D node-map field (field.py:101-560 API)."""

    def __init__(self, label="Field", dim=0, field=None, scaling=1.0, units="m", debug=False,
                 method="linear", interpolator_backend="auto"):
        if units not in UNIT_SCALES:
            raise ValueError(f"Unknown unit '{units}'. Must be one of {list(UNIT_SCALES.keys())}")
        self._label = label
        self._dim = dim
        self._scaling = scaling
        self._debug = debug
        self._filename = None
        self._metadata = {}
        self._interpolator_backend = interpolator_backend
        self._method = method
        # like the reference, _unit_scale is stored but never applied (field.py:157)
        self._unit_scale = UNIT_SCALES[units]
        self._field = {"x": None, "y": None, "z": None} if field is None else field

    def __call__(self, pts):
        pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
        if pts.shape[1] != 3:
            raise ValueError(f"Points must have shape (M, 3), got {pts.shape}")
        if self._dim == 0:
            m = pts.shape[0]
            return np.column_stack([self._scaling * self._field[c] * np.ones(m) for c in "xyz"])
        if self._dim not in (1, 2, 3):
            raise NotImplementedError(f"{self._dim}D fields are not supported by this package")
        return _evaluate(self, pts)

    def __str__(self):
        if self._dim == 0:
            return f"Field '{self._label}' (0D constant): {[self._field[k] for k in 'xyz']}"
        return f"Field '{self._label}' ({self._dim}D interpolated)"

    def __repr__(self):
        return f"Field(label='{self._label}', dim={self._dim}, scaling={self._scaling})"

    @classmethod
    def from_arrays(cls, grid, values, **kwargs):
        """Field on a rectilinear node grid (field.py:345-387).  ``values``
        components may be None (identically zero)."""
        field = cls(**kwargs)
        points = [np.asarray(grid[k], dtype=np.float64) for k in "xyz" if k in grid and len(grid[k]) > 1]
        field._dim = len(points)
        for c in "xyz":
            if values.get(c) is not None:
                field._field[c] = get_interpolator(tuple(points), values[c], method=field._method,
                                                   bounds_error=False, fill_value=0.0,
                                                   backend=field._interpolator_backend)
        return field

    @classmethod
    def from_file(cls, filename, **kwargs):
        """Field from a map file, the format chosen by extension (field.py:284-343):
        .table OPERA, .comsol COMSOL, .dat OPAL midplane, .map AIMA AGORA,
        .h5/.h5part H5Part, .pickle a saved Field.  As in the reference,
        ``kwargs`` go to the constructor, not to the loader."""
        from . import loaders
        if not os.path.exists(filename):
            raise FileNotFoundError(f"Field file not found: {filename}")
        ext = os.path.splitext(filename)[1]
        field = cls(**kwargs)
        field._filename = filename
        if ext == ".pickle":
            field._load_pickle(filename)
            return field
        if ext not in loaders.LOADERS:
            raise ValueError(f"Unknown file extension: {ext}")
        data = loaders.LOADERS[ext](filename)
        points = [data["grid"][k] for k in "xyz" if k in data["grid"] and len(data["grid"][k]) > 1]
        field._dim = data["dim"]
        field._metadata = data["metadata"]
        for c in "xyz":
            if c in data["values"]:
                field._field[c] = get_interpolator(tuple(points), data["values"][c], method=field._method,
                                                   bounds_error=False, fill_value=0.0,
                                                   backend=field._interpolator_backend)
        return field

    def _load_pickle(self, filename):
        """Restore a Field saved by ``save_pickle`` (field.py:510-518)."""
        with open(filename, "rb") as fh:
            data = pickle.load(fh)
        for key in ("_label", "_dim", "_scaling", "_field", "_unit_scale", "_metadata"):
            if key in data:
                setattr(self, key, data[key])

    def save_pickle(self, filename):
        """Save the Field's attributes (field.py:520-534)."""
        data = {"_label": self._label, "_dim": self._dim, "_scaling": self._scaling, "_field": self._field,
                "_unit_scale": self._unit_scale, "_metadata": self._metadata}
        with open(filename, "wb") as fh:
            pickle.dump(data, fh)

    @classmethod
    def zero(cls, dim=3):
        """Zero field (field.py:389-407)."""
        if dim == 0:
            return cls(label="Zero Field", dim=0, field={"x": 0.0, "y": 0.0, "z": 0.0})
        grid = tuple(np.array([-1e20, 1e20]) for _ in range(dim))
        f = cls(label="Zero Field", dim=dim)
        for c in "xyz":
            f._field[c] = CudaInterpolator(grid, np.zeros([2] * dim), bounds_error=False, fill_value=0.0)
        return f

    @property
    def label(self):
        return self._label

    @label.setter
    def label(self, value):
        self._label = value

    @property
    def dim(self):
        return self._dim

    @property
    def scaling(self):
        return self._scaling

    @scaling.setter
    def scaling(self, value):
        self._scaling = value

    @property
    def metadata(self):
        return self._metadata


class CompositeField(FieldBase):
    """sum_i w_i F_i (field.py:595-658)."""

    def __init__(self, fields, weights):
        if len(fields) != len(weights):
            raise ValueError("Number of fields must match number of weights")
        self.fields = list(fields)
        self.weights = np.array(weights, dtype=np.float64)
        self.n_fields = len(fields)

    def __call__(self, pts):
        return _evaluate(self, pts)

    def __str__(self):
        return f"CompositeField with {len(self.fields)} components"


class ScaledField(FieldBase):
    """scale * F + offset (field.py:661-690)."""

    def __init__(self, field, scale=1.0, offset=0.0):
        self.field = field
        self.scale = scale
        self.offset = offset

    def __call__(self, pts):
        return _evaluate(self, pts)


class FieldMap:
    """E and B container; missing fields are zero (field.py:697-755)."""

    def __init__(self, efield=None, bfield=None, metadata=None):
        self.efield = efield if efield is not None else Field.zero()
        self.bfield = bfield if bfield is not None else Field.zero()
        self.metadata = metadata if metadata is not None else {}

    @classmethod
    def from_fields(cls, efield, bfield, **metadata):
        return cls(efield=efield, bfield=bfield, metadata=metadata)

    def __str__(self):
        return f"FieldMap(E: {self.efield}, B: {self.bfield})"


class CudaInterpolator:
    """Linear / bilinear / trilinear interpolation of one component on the
    GPU (the 'cuda' backend of ``get_interpolator``; the API of
    ``NumbaInterpolator``, field_src/interpolators.py:273-408, 1 to 3 axes)."""

    def __init__(self, points, values, method="linear", bounds_error=True, fill_value=np.nan):
        if method != "linear":
            raise ValueError(f"Method '{method}' not supported. Use 'linear'")
        self.ndim = len(points)
        if self.ndim not in (1, 2, 3):
            raise ValueError(f"Only 1D, 2D, 3D supported. Got {self.ndim}D")
        self.method = method
        self.bounds_error = bounds_error
        self.fill_value = float(fill_value)
        self._grid = tuple(np.ascontiguousarray(p, dtype=np.float64) for p in points)
        if type(values).__module__.startswith("torch"):
            # device node values (e.g. a space-charge field): kept on the device
            import torch
            self._values = values.to(torch.float32 if values.dtype == torch.float32 else torch.float64).contiguous()
        else:
            vals = np.asarray(values)
            self._values = np.ascontiguousarray(vals, dtype=np.float32 if vals.dtype == np.float32 else np.float64)
        self._bounds = tuple((float(g[0]), float(g[-1])) for g in self._grid)
        expected = tuple(len(g) for g in self._grid)
        if tuple(self._values.shape) != expected:
            raise ValueError(f"Values shape {self._values.shape} does not match grid shape {expected}")

    def __call__(self, xi, method=None):
        xi = np.asarray(xi, dtype=np.float64)
        single = xi.ndim == 1
        if single:
            xi = xi.reshape(1, -1)
        if xi.shape[1] != self.ndim:
            raise ValueError(f"Points have dimension {xi.shape[1]}, expected {self.ndim}")
        if self.bounds_error:
            for i, (lo, hi) in enumerate(self._bounds):
                if np.any(xi[:, i] < lo) or np.any(xi[:, i] > hi):
                    raise ValueError("One or more points are outside the interpolation domain")
        # a one-component Field of the same dimension: its 1D axis is z, its
        # 2D axes are x and y (field.py:457-489)
        pts = np.zeros((xi.shape[0], 3))
        if self.ndim == 1:
            pts[:, 2] = xi[:, 0]
        else:
            pts[:, :self.ndim] = xi
        one = Field(dim=self.ndim, field={"x": _Plain(self), "y": None, "z": None})
        out = _evaluate(one, pts)[:, 0]
        if self.fill_value != 0.0:
            outside = np.zeros(xi.shape[0], dtype=bool)
            for i, (lo, hi) in enumerate(self._bounds):
                outside |= (xi[:, i] < lo) | (xi[:, i] > hi)
            out[outside] = self.fill_value
        if single:
            return float(out[0])
        return out


class _Plain:
    """The node data of a CudaInterpolator with fill 0 (what the kernel does)."""

    def __init__(self, interp):
        self._grid = interp._grid
        self._values = interp._values
        self.fill_value = 0.0
        self.method = "linear"


def get_interpolator(points, values, method="linear", bounds_error=False, fill_value=0.0, backend="auto"):
    """Factory with the reference's signature (interpolators.py:533-610).
    'auto' and 'cuda' give the GPU interpolator; the CPU backends of the
    reference are not part of this package."""
    backend = backend.lower()
    if backend in ("auto", "cuda"):
        return CudaInterpolator(points, values, method, bounds_error, fill_value)
    if backend in ("numba", "fast", "scipy", "cupy"):
        raise NotImplementedError(f"backend {backend!r} is a CPU backend of the reference; this package "
                                  "evaluates fields on the GPU ('cuda')")
    raise ValueError(f"Unknown backend '{backend}'. Use: 'auto', 'cuda'")
