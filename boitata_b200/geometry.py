"""Block-model geometry as kriging targets.

Mirrors crates/core/src/block_model.rs:19-86 (Geometry: corner origin, cell
size, cell count, azimuth/dip/rake; cells x fastest, then y, then z) and
BlockModel::centroids (:431-445) for a regular model. The engine generates
the centroids on the device, in the reference's arithmetic order.
"""

import math

import numpy as np

from . import _native as N
from .errors import InvalidInput


class Geometry:
    def __init__(self, origin, size, count, rotation=(0.0, 0.0, 0.0)):
        self.origin = tuple(float(v) for v in origin)
        self.size = tuple(float(v) for v in size)
        self.count = tuple(int(v) for v in count)
        self.rotation = tuple(float(v) for v in rotation)
        # block_model.rs:29-56
        if len(self.origin) != 3 or len(self.size) != 3 or len(self.count) != 3 or len(self.rotation) != 3:
            raise InvalidInput("origin, size, count and rotation need 3 values each")
        if any(not (math.isfinite(s) and s > 0) for s in self.size):
            raise InvalidInput("cell sizes must be positive")
        if any(c <= 0 for c in self.count):
            raise InvalidInput("cell counts must be positive")
        if any(not math.isfinite(v) for v in self.origin + self.rotation):
            raise InvalidInput("origin and rotation must be finite")

    def cells(self):
        return self.count[0] * self.count[1] * self.count[2]

    def to_c(self):
        g = N.GeometryC()
        for a in range(3):
            g.origin[a], g.size[a], g.count[a], g.rotation[a] = self.origin[a], self.size[a], self.count[a], \
                self.rotation[a]
        return g

    def __repr__(self):
        return f"Geometry(origin={self.origin}, size={self.size}, count={self.count}, rotation={self.rotation})"


class _Columns:
    """Named attribute columns of a container, one value a row (containers.rs:75-210: attributes,
    `container[name]`, with_column)."""

    def _set_columns(self, attributes, rows):
        cols = {}
        if attributes is not None:
            names = list(attributes.column_names) if hasattr(attributes, "column_names") else list(attributes)
            for name in names:
                a = np.asarray(attributes[name])
                if a.ndim != 1 or len(a) != rows:
                    raise InvalidInput(f'column "{name}": expected {rows} values, got shape {a.shape}')
                cols[str(name)] = a
        self.attributes = cols

    @property
    def column_names(self):
        return list(self.attributes)

    def __contains__(self, name):
        return name in self.attributes

    def __getitem__(self, name):
        try:
            return self.attributes[name]
        except KeyError:
            import difflib

            from .errors import MissingColumn

            close = difflib.get_close_matches(str(name), self.column_names, n=1)
            hint = f' (did you mean "{close[0]}"?)' if close else ""
            raise MissingColumn(f'no column "{name}"{hint}; columns: {", ".join(self.column_names)}') from None

    def with_column(self, name, values):
        """A copy with the column `name` added or replaced."""
        import copy

        out = copy.copy(self)
        out.attributes = dict(self.attributes)
        a = np.asarray(values)
        if a.ndim != 1 or len(a) != len(self):
            raise InvalidInput(f'column "{name}": expected {len(self)} values, got shape {a.shape}')
        out.attributes[str(name)] = a
        return out


class PointSet(_Columns):
    """Points with attribute columns: PointSet(coords, attributes=None, *, crs=None, length_unit=None) as the
    reference's (crates/py/src/containers.rs:75-100); `coords` (n, 2) or (n, 3), 2-D points on z = 0."""

    def __init__(self, coords, attributes=None, *, crs=None, length_unit=None):
        a = np.asarray(coords, dtype=np.float64)
        if a.ndim != 2 or a.shape[1] not in (2, 3):
            raise InvalidInput("coordinates must be a 2-D array of shape (n, 2) or (n, 3)")
        if not np.all(np.isfinite(a)):
            raise InvalidInput("coordinates must be finite")
        if a.shape[1] == 2:
            a = np.column_stack([a, np.zeros(len(a))])
        self._coords = np.ascontiguousarray(a)
        self._set_columns(attributes, len(a))
        self.crs, self.length_unit = crs, length_unit

    @property
    def coords(self):
        return self._coords

    def __len__(self):
        return len(self._coords)


class BlockModel(_Columns):
    """A regular block model: its `geometry` and the centroids of its cells.

    BlockModel(origin, size, count, *, rotation=(0, 0, 0)) as the reference's
    constructor (crates/py/src/containers.rs:788-840: `origin` the corner of
    the first cell, `rotation` azimuth, dip, rake in degrees), or
    BlockModel(geometry). Masked models (`index`) are not run here.
    """

    def __init__(self, origin, size=None, count=None, *, rotation=(0.0, 0.0, 0.0), attributes=None, index=None,
                 crs=None, length_unit=None):
        from .errors import Unsupported

        if index is not None:
            raise Unsupported("masked block models (index) are not run by this engine")
        if isinstance(origin, Geometry):
            if size is not None or count is not None:
                raise InvalidInput("give a Geometry, or origin, size and count")
            self.geometry = origin
        elif size is None or count is None:
            raise InvalidInput("BlockModel needs origin, size and count, or a Geometry")
        else:
            # Two values stand for x and y: z takes origin 0, size 1, count 1 (containers.rs:804-806).
            pad = lambda v, fill: tuple(v) + (fill,) if len(tuple(v)) == 2 else tuple(v)  # noqa: E731
            self.geometry = Geometry(pad(origin, 0.0), pad(size, 1.0), pad(count, 1), rotation)
        self._set_columns(attributes, self.geometry.cells())
        self.crs, self.length_unit = crs, length_unit

    @property
    def origin(self):
        return self.geometry.origin

    @property
    def size(self):
        return self.geometry.size

    @property
    def count(self):
        return self.geometry.count

    @property
    def rotation(self):
        return self.geometry.rotation

    @property
    def coords(self):
        """Every cell's centroid, (n, 3) in cell order, computed by the engine."""
        return self.centroids()

    def __len__(self):
        return self.geometry.cells()

    def centroids(self, context=None, first=0, count=None):
        """Centroids (count, 3) of cells first .. first + count - 1 (all by default), cell order, computed by
        the engine on the device (block_model.rs:431-445: row index i + nx (j + ny k))."""
        import ctypes

        from ._native import Context

        ctx = context or Context()
        n = self.geometry.cells()
        count = n - first if count is None else count
        if first < 0 or count < 0 or first + count > n:
            raise InvalidInput("the cell range must lie within the block model")
        out = np.empty((count, 3), dtype=np.float64)
        g = self.geometry.to_c()
        rc = ctx._lib.btk_centroids(ctx.handle, ctypes.byref(g), first, count, out.ctypes.data)
        ctx.check(rc, "centroids")
        return out
