"""Turn reference-style field objects into device field maps.

The pusher's field protocol is the reference's: a callable ``(M,3) -> (M,3)``
(src/PyPATools/field.py:72-86).  To evaluate fields inside the GPU kernels
the callable must be one whose values are data, not code.  Accepted (this
package's classes and the reference's own, by duck typing):

* ``Field`` of dim 0 (constant, ``_field`` holds numbers, field.py:441-455);
* ``Field`` of dim 3 whose component interpolators expose a node grid and
  values: ``NumbaInterpolator`` / ``CoordinateMapper`` (``_grid``,
  ``_values``), scipy ``RegularGridInterpolator`` (``grid``, ``values``),
  this package's ``CudaInterpolator``; the field's ``_scaling`` multiplies
  them (field.py:491-504);
* ``Field`` of dim 1 or 2 with such interpolators: a dim-1 field varies
  along z only and a dim-2 field along x and y, whatever axes its grid was
  given on (``_get_field_1d`` / ``_get_field_2d`` evaluate the interpolators
  at ``pts[:, 2]`` and ``pts[:, :2]``, field.py:457-489); it becomes a map
  with one-node axes, which the kernels treat as unbounded and constant;
* ``Field.zero()`` (field.py:389-407) -> nothing;
* ``ScaledField`` (scale * F + offset, field.py:661-690);
* ``CompositeField`` (sum of w_i F_i, field.py:595-658);
* ``None`` -> zero field.

Anything else raises ``NotImplementedError``: there is no CPU fallback.

Terms on the same node grid are summed into one device map; when E and B
share a grid they share one map, so each step does one cell lookup and one
gather of [E | B] node records.  Components that are identically zero in
every term (an RF gap's Ex, Ey, Bx, By; a sector magnet's Bx, By) are not
stored: the map's records keep only the others (``ppt_fieldmap_create_masked``),
which the kernels then neither gather nor multiply.
"""
import weakref

import numpy as np

from . import _lib


class _MapTerm:
    __slots__ = ("grid", "comps", "scale")

    def __init__(self, grid, comps, scale):
        self.grid = grid            # tuple of 3 float64 arrays
        self.comps = comps          # {'x','y','z'} -> ndarray (float32/float64) or None
        self.scale = scale          # float


def check_term_sizes(term):
    """Every component of a map term holds one value per grid node: the map
    add kernel reads that many from each component's data pointer, so a
    shorter array (an interpolator built elsewhere, a mutated tensor) is
    refused here instead of read past its end."""
    nodes = 1
    for axis in term.grid:
        nodes *= int(np.asarray(axis).shape[0])
    for c, a in term.comps.items():
        if a is None:
            continue
        size = int(a.numel()) if _is_tensor(a) else int(np.asarray(a).size)
        if size != nodes:
            dims = " x ".join(str(int(np.asarray(ax).shape[0])) for ax in term.grid)
            raise ValueError(f"field component {c!r} has {size} node values, its grid {dims} = {nodes} nodes")


class FieldTerms:
    """A field as (constant vector, list of map terms)."""

    def __init__(self):
        self.const = np.zeros(3)
        self.terms = []

    def scaled(self, s):
        out = FieldTerms()
        out.const = self.const * s
        out.terms = [_MapTerm(t.grid, t.comps, t.scale * s) for t in self.terms]
        return out

    def add(self, other, w=1.0):
        self.const = self.const + w * other.const
        self.terms += [_MapTerm(t.grid, t.comps, t.scale * w) for t in other.terms]


def _interp_grid_values(interp):
    """Node grid and values of one component interpolator, or None for a
    zero-valued one."""
    if interp is None:
        return None
    if hasattr(interp, "_grid") and hasattr(interp, "_values"):
        grid, values = interp._grid, interp._values
    elif hasattr(interp, "grid") and hasattr(interp, "values"):
        grid, values = interp.grid, interp.values
    else:
        raise NotImplementedError(
            f"cannot read node values from interpolator of type {type(interp).__name__}")
    fill = getattr(interp, "fill_value", 0.0)
    if fill is not None and fill != 0.0:
        raise NotImplementedError("only fill_value=0.0 (the Field default) is supported on the GPU")
    method = getattr(interp, "method", "linear")
    if method != "linear":
        raise NotImplementedError(f"interpolation method {method!r}: only 'linear' runs on the GPU")
    return tuple(np.asarray(g, dtype=np.float64) for g in grid), values


_zero_cache = {}


def _is_tensor(a):
    return type(a).__module__.startswith("torch") and hasattr(a, "data_ptr")


def _all_zero(values):
    """True when a node array is identically zero.  Remembered per array
    object (validated through a weak reference, so an array allocated later
    at a freed one's address is scanned afresh); numpy node arrays are
    treated as immutable once a field uses them, torch tensors are rescanned
    after an in-place change (their version counter)."""
    if _is_tensor(values):
        key = (id(values), values._version)
        hit = _zero_cache.get(key)
        if hit is not None and hit[0]() is values:
            return hit[1]
        result = not bool(values.any())
        _zero_cache[key] = (weakref.ref(values), result)
        return result
    a = np.asarray(values)
    key = id(a)
    hit = _zero_cache.get(key)
    if hit is not None and hit[0]() is a:
        return hit[1]
    result = not np.any(a)
    try:
        ref = weakref.ref(a)
    except TypeError:
        return result
    if len(_zero_cache) > 4096:
        _zero_cache.clear()
    _zero_cache[key] = (ref, result)
    return result


_ONE_NODE = np.zeros(1)


def _as_3d(grid):
    """The grid of a 1D (z) or 2D (x, y) interpolator as a 3D node grid whose
    other axes have one node (field.py:457-489).  The node values keep their
    shape: flattened in C order they are already the 3D map's [i][j][k]."""
    if len(grid) == 1:
        return (_ONE_NODE, _ONE_NODE, grid[0])
    if len(grid) == 2:
        return (grid[0], grid[1], _ONE_NODE)
    return grid


def decompose(field):
    """Field-like object -> FieldTerms."""
    out = FieldTerms()
    if field is None:
        return out
    # this package's and the reference's ScaledField / CompositeField
    if hasattr(field, "field") and hasattr(field, "scale") and hasattr(field, "offset"):
        inner = decompose(field.field).scaled(float(field.scale))
        off = np.broadcast_to(np.asarray(field.offset, dtype=np.float64), (3,))
        inner.const = inner.const + off
        return inner
    if hasattr(field, "fields") and hasattr(field, "weights"):
        for f, w in zip(field.fields, np.asarray(field.weights, dtype=np.float64)):
            out.add(decompose(f), float(w))
        return out
    if hasattr(field, "_dim") and hasattr(field, "_field"):
        dim = field._dim
        scaling = float(getattr(field, "_scaling", 1.0))
        comps = field._field
        if dim == 0:
            out.const = scaling * np.array([float(comps[c] or 0.0) for c in "xyz"])
            return out
        if dim not in (1, 2, 3):
            raise NotImplementedError(f"{dim}D fields are not on the GPU path")
        grid = None
        values = {}
        for c in "xyz":
            gv = _interp_grid_values(comps.get(c))
            if gv is None:
                values[c] = None
                continue
            g, v = gv
            if len(g) != dim:
                raise NotImplementedError(f"a {dim}D field needs {dim}D component interpolators")
            g = _as_3d(g)
            if grid is None:
                grid = g
            elif not all(np.array_equal(a, b) for a, b in zip(grid, g)):
                raise NotImplementedError("components of one Field on different grids")
            values[c] = v
        if grid is None:
            return out
        # Field.zero(): all-zero node values contribute nothing anywhere
        if all(values[c] is None or _all_zero(values[c]) for c in "xyz"):
            return out
        out.terms.append(_MapTerm(grid, values, scaling))
        return out
    raise NotImplementedError(
        f"field of type {type(field).__name__} cannot be evaluated on the GPU: pass a Field "
        "(dim 0 to 3), ScaledField or CompositeField built from node maps")


def _grid_key(grid):
    return tuple((g.shape[0], float(g[0]), float(g[-1]), hash(g.tobytes())) for g in grid)


class DeviceFields:
    """Device maps + constants for one (efield, bfield, precision) triple."""

    def __init__(self, efield, bfield, precision="fp64", device=None, prune=True):
        import torch
        self._torch = torch
        lib = _lib.load()
        self.precision = precision
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        store = _lib.DTYPE_F64 if precision == "fp64" else _lib.DTYPE_F32
        e_terms, b_terms = decompose(efield), decompose(bfield)
        groups = {}   # grid key -> dict(grid, e=[terms], b=[terms])
        for kind, ft in (("e", e_terms), ("b", b_terms)):
            for t in ft.terms:
                key = _grid_key(t.grid)
                g = groups.setdefault(key, {"grid": t.grid, "e": [], "b": []})
                g[kind].append(t)
        if len(groups) > _lib.MAX_MAPS:
            raise NotImplementedError(f"at most {_lib.MAX_MAPS} distinct node grids per pusher call")
        self.maps = []
        self.layouts = []
        self.map_bytes = 0
        self.n_components = 0
        has_const = bool(np.any(e_terms.const != 0.0) or np.any(b_terms.const != 0.0))
        with torch.cuda.device(self.device):
            stream = _lib.stream_handle()
            for g in groups.values():
                mask = 0
                for kind, base in (("e", 0), ("b", 3)):
                    for t in g[kind]:
                        for ci, c in enumerate("xyz"):
                            a = t.comps.get(c)
                            if a is not None and not _all_zero(a):
                                mask |= 1 << (base + ci)
                if mask == 0:
                    continue     # every term of this grid is zero
                if not prune:
                    mask = (0x07 if g["e"] else 0) | (0x38 if g["b"] else 0)
                if precision == "mixed" and has_const:
                    mask = _lib.FULL_MASK   # the mixed kernels take constant parts with this layout only
                handle = ctypes_void()
                desc = _lib.GridDesc()
                axes = [np.ascontiguousarray(a, dtype=np.float64) for a in g["grid"]]
                for d in range(3):
                    desc.n[d] = axes[d].shape[0]
                    desc.axis[d] = axes[d].ctypes.data
                _lib.check(lib.ppt_fieldmap_create_masked(desc, mask, store, handle))
                self.maps.append(handle.value)
                for kind in ("e", "b"):
                    for t in g[kind]:
                        self._add_term(lib, handle.value, kind, t, stream, mask)
                nbytes, flags = _lib.c_int64(), _lib.c_int()
                _lib.check(lib.ppt_fieldmap_info(handle.value, nbytes, flags))
                self.map_bytes += nbytes.value
                self.layouts.append((flags.value >> 8) & 0x3F)
                self.n_components += bin(mask).count("1")
            torch.cuda.current_stream().synchronize()
        self.fields = _lib.Fields()
        for i, h in enumerate(self.maps):
            self.fields.maps[i] = h
        self.fields.n_maps = len(self.maps)
        for c in range(3):
            self.fields.e_const[c] = float(e_terms.const[c])
            self.fields.b_const[c] = float(b_terms.const[c])
        self.e_const = e_terms.const.copy()
        self.b_const = b_terms.const.copy()
        self._finalizer = weakref.finalize(self, _destroy_maps, list(self.maps))

    def _add_term(self, lib, handle, kind, term, stream, mask):
        torch = self._torch
        check_term_sizes(term)
        ptrs = (_lib.c_void_p * 6)()
        scales = (_lib.c_double * 6)()
        base = 0 if kind == "e" else 3
        # components outside the mask are identically zero: nothing to add
        present = [(ci, term.comps[c] if _is_tensor(term.comps[c]) else np.asarray(term.comps[c]))
                   for ci, c in enumerate("xyz") if term.comps.get(c) is not None and mask & (1 << (base + ci))]
        if not present:
            return
        # float32 node values stay float32 (exact); anything else goes as float64
        all_f32 = all(str(a.dtype) in ("float32", "torch.float32") for _, a in present)
        np_dtype, src_dtype = (np.float32, _lib.DTYPE_F32) if all_f32 else (np.float64, _lib.DTYPE_F64)
        t_dtype = torch.float32 if all_f32 else torch.float64
        keep = []
        for ci, a in present:
            if _is_tensor(a):
                # device node values (a space-charge field) go straight into the map
                tdev = a.to(device=self.device, dtype=t_dtype).contiguous()
            else:
                tdev = torch.from_numpy(np.ascontiguousarray(a, dtype=np_dtype)).to(self.device)
            keep.append(tdev)
            slot = ci + (0 if kind == "e" else 3)
            ptrs[slot] = tdev.data_ptr()
            scales[slot] = float(term.scale)
        _lib.check(lib.ppt_fieldmap_add(handle, ptrs, scales, src_dtype, stream))
        torch.cuda.current_stream().synchronize()   # keep the sources alive until the adds ran

    @property
    def has_maps(self):
        return bool(self.maps)


def ctypes_void():
    return _lib.c_void_p()


def _destroy_maps(handles):
    try:
        lib = _lib.load()
    except ImportError:
        return
    for h in handles:
        if h:
            lib.ppt_fieldmap_destroy(h)


class FieldCache:
    """Re-use device maps while the field objects and their scalings are
    unchanged (the reference re-evaluates the Python callables every step;
    here the maps are uploaded once)."""

    def __init__(self, capacity=4):
        self.capacity = capacity
        self._entries = []   # (key, refs, DeviceFields)

    @staticmethod
    def _fingerprint(field):
        ft = decompose(field)

        def ident(a):   # a torch tensor changed in place is a new field
            return (id(a), a._version) if _is_tensor(a) else id(a)
        return (tuple(ft.const.tolist()),
                tuple((ident(t.comps.get("x")), ident(t.comps.get("y")), ident(t.comps.get("z")), t.scale)
                      for t in ft.terms))

    def get(self, efield, bfield, precision, device=None):
        key = (id(efield), id(bfield), precision, str(device),
               self._fingerprint(efield), self._fingerprint(bfield))
        for i, (k, refs, df) in enumerate(self._entries):
            if k == key and all(r() is not None for r in refs):
                self._entries.insert(0, self._entries.pop(i))
                return df
        df = DeviceFields(efield, bfield, precision, device)
        refs = []
        for f in (efield, bfield):
            try:
                refs.append(weakref.ref(f) if f is not None else (lambda: True))
            except TypeError:
                refs.append(lambda: True)
        self._entries.insert(0, (key, refs, df))
        del self._entries[self.capacity:]
        return df
