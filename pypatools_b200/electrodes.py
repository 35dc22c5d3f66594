"""Electrode surfaces: particles whose step crosses them stop.

The reference's ``Pusher(..., electrode_assembly=...)`` takes a
``PyElectrodeAssembly`` (the external py_electrodes package) and, after every
step of ``track_batch``, deactivates the particles whose step segment meets an
electrode (``segment_intersects_surface(r_old, r_new)["hit_mask"]``,
src/PyPATools/pusher.py:982-990).  Here an electrode assembly is a triangle
mesh on the GPU (``ppt_surface_*``): ``ElectrodeSurface`` wraps one, offers the
same ``segment_intersects_surface`` call, and ``PusherGPU`` runs the test
inside the float64 track kernel, step by step.

``PusherGPU`` accepts an ``ElectrodeSurface`` or any object with ``vertices``
((V, 3) float) and ``triangles`` ((T, 3) int) arrays describing the electrode
surfaces.  The builders below make the simple shapes of beam-line tests: an
aperture plate (an annulus in a z plane), a tube (a cylinder along z), and a
closed annular cylinder (a thick pipe or plate, for the space-charge solver's
conductor cells, which need closed surfaces).
"""
import ctypes
import math

import numpy as np

from . import _lib


class ElectrodeSurface:
    """A triangle mesh of electrode surfaces (metres)."""

    def __init__(self, vertices, triangles):
        v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64))
        t = np.ascontiguousarray(np.asarray(triangles, dtype=np.int64))
        if v.ndim != 2 or v.shape[1] != 3 or t.ndim != 2 or t.shape[1] != 3:
            raise ValueError("vertices must be (V, 3) and triangles (T, 3)")
        if t.size and (t.min() < 0 or t.max() >= v.shape[0]):
            raise ValueError("triangle vertex index out of range")
        self.vertices = v
        self.triangles = t
        self._handles = {}   # device index -> ppt_surface*

    @classmethod
    def from_assembly(cls, assembly):
        """An ElectrodeSurface from this class or an object exposing
        ``vertices`` and ``triangles``."""
        if isinstance(assembly, cls):
            return assembly
        if hasattr(assembly, "vertices") and hasattr(assembly, "triangles"):
            return cls(assembly.vertices, assembly.triangles)
        raise NotImplementedError(
            f"electrode assembly of type {type(assembly).__name__}: the GPU path needs its surfaces as a "
            "triangle mesh (an ElectrodeSurface, or an object with 'vertices' and 'triangles')")

    def __add__(self, other):
        other = ElectrodeSurface.from_assembly(other)
        return ElectrodeSurface(np.concatenate([self.vertices, other.vertices]),
                                np.concatenate([self.triangles, other.triangles + self.vertices.shape[0]]))

    def handle(self, device):
        """The device copy (created on first use on ``device``)."""
        import torch
        dev = torch.device(device)
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        h = self._handles.get(idx)
        if h is None:
            lib = _lib.load()
            out = ctypes.c_void_p()
            with torch.cuda.device(idx):
                _lib.check(lib.ppt_surface_create(self.vertices.shape[0], self.vertices.ctypes.data,
                                                  self.triangles.shape[0], self.triangles.ctypes.data, out))
            h = out.value
            self._handles[idx] = h
        return h

    def info(self, device="cuda"):
        nbytes = ctypes.c_int64()
        dims = (ctypes.c_int32 * 3)()
        _lib.check(_lib.load().ppt_surface_info(self.handle(device), nbytes, dims))
        return {"bytes": nbytes.value, "cells": tuple(dims)}

    def segment_intersects_surface(self, p0, p1, device="cuda"):
        """For each row, does the segment p0 -> p1 meet the surface?  Returns
        ``{"hit_mask": bool (M,)}``, the key the reference reads
        (pusher.py:984-986)."""
        import torch
        a = np.ascontiguousarray(np.asarray(p0, dtype=np.float64).reshape(-1, 3))
        b = np.ascontiguousarray(np.asarray(p1, dtype=np.float64).reshape(-1, 3))
        if a.shape != b.shape:
            raise ValueError("p0 and p1 must have the same shape")
        m = a.shape[0]
        if m == 0:
            return {"hit_mask": np.zeros(0, dtype=bool)}
        dev = torch.device(device)
        h = self.handle(dev)
        da, db = torch.from_numpy(a).to(dev), torch.from_numpy(b).to(dev)
        hit = torch.empty(m, dtype=torch.uint8, device=dev)
        with torch.cuda.device(da.device):
            _lib.check(_lib.load().ppt_surface_segments_hit(h, m, da.data_ptr(), db.data_ptr(), hit.data_ptr(),
                                                            _lib.stream_handle()))
        return {"hit_mask": hit.cpu().numpy().astype(bool)}

    def __del__(self):
        handles, self._handles = getattr(self, "_handles", {}), {}
        if not handles:
            return
        try:
            lib = _lib.load()
        except ImportError:
            return
        for h in handles.values():
            lib.ppt_surface_destroy(h)

    # -- simple shapes --------------------------------------------------------
    @classmethod
    def aperture_plate(cls, z, r_hole, r_outer, n_phi=64, n_r=4):
        """An annulus r_hole <= r <= r_outer in the plane at z (a plate with a
        round hole), n_phi segments around, n_r rings across."""
        phi = np.linspace(0.0, 2.0 * math.pi, n_phi, endpoint=False)
        radii = np.linspace(r_hole, r_outer, n_r + 1)
        verts = np.array([[r * math.cos(p), r * math.sin(p), z] for r in radii for p in phi])
        tris = []
        for i in range(n_r):
            for j in range(n_phi):
                a, b = i * n_phi + j, i * n_phi + (j + 1) % n_phi
                c, d = a + n_phi, b + n_phi
                tris += [[a, b, d], [a, d, c]]
        return cls(verts, np.array(tris))

    @classmethod
    def annular_cylinder(cls, r_in, r_out, z0, z1, n_phi=64, n_z=16, n_r=2):
        """A closed solid: the ring r_in <= r <= r_out, z0 <= z <= z1 (a thick
        beam pipe, or a thick aperture plate when z1 - z0 is small).  Its
        surface is closed, so rays from inside the solid cross it an odd number
        of times (the conductor test of the space-charge solver); the other
        builders make open sheets, enough for stopping particles."""
        return (cls.tube(r_out, z0, z1, n_phi, n_z) + cls.tube(r_in, z0, z1, n_phi, n_z) +
                cls.aperture_plate(z0, r_in, r_out, n_phi, n_r) + cls.aperture_plate(z1, r_in, r_out, n_phi, n_r))

    @classmethod
    def tube(cls, radius, z0, z1, n_phi=64, n_z=16):
        """A cylinder of the given radius along z from z0 to z1 (a beam pipe)."""
        phi = np.linspace(0.0, 2.0 * math.pi, n_phi, endpoint=False)
        zs = np.linspace(z0, z1, n_z + 1)
        verts = np.array([[radius * math.cos(p), radius * math.sin(p), z] for z in zs for p in phi])
        tris = []
        for i in range(n_z):
            for j in range(n_phi):
                a, b = i * n_phi + j, i * n_phi + (j + 1) % n_phi
                c, d = a + n_phi, b + n_phi
                tris += [[a, b, d], [a, d, c]]
        return cls(verts, np.array(tris))
