"""Search neighbourhood parameters, as the reference's `Search` takes them.

Mirrors crates/py/src/estimation.rs:414-510 (constructor) and
crates/estimation/src/search.rs:31-81, 185-264 (fields, defaults, check).
"""

import math

from . import _native as N
from .errors import InvalidInput
from .variogram import aniso_c, anisotropy


def _count(v, what):
    if v is None:
        return None
    if isinstance(v, bool) or int(v) != v or v < 0:
        raise InvalidInput(f"{what} must be a non-negative integer")
    return int(v)


class Search:
    """Neighbourhood of each target: radius (major-axis metres of the ellipsoid), sample counts, octants."""

    def __init__(self, radius=None, *, max_samples=16, min_samples=1, octant=False, sectors=None,
                 max_per_sector=None, max_per_hole=None, rotation=None, ratios=None, ranges=None,
                 min_sectors=None, max_empty_sectors=None, min_holes=None, target_slope=None,
                 target_efficiency=None):
        # crates/py/src/estimation.rs:458-473: at most one calibration target.
        if target_slope is not None and target_efficiency is not None:
            raise InvalidInput("give at most one of target_slope and target_efficiency")
        if target_slope is not None and not (math.isfinite(float(target_slope)) and float(target_slope) > 0.0):
            raise InvalidInput("target_slope must be finite and > 0")
        if target_efficiency is not None and not (math.isfinite(float(target_efficiency)) and
                                                  float(target_efficiency) <= 1.0):
            raise InvalidInput("target_efficiency must be finite and <= 1")
        self.target_slope = None if target_slope is None else float(target_slope)
        self.target_efficiency = None if target_efficiency is None else float(target_efficiency)
        if radius is not None and ranges is not None:
            raise InvalidInput("give radius or ranges, not both")
        if radius is None and ranges is None:
            raise InvalidInput("give radius or ranges")
        if ranges is not None:
            if ratios is not None:
                raise InvalidInput("give ratios with radius, not with ranges")
            major, semi, minor = (float(r) for r in ranges)
            if not (major > 0 and semi > 0 and minor > 0):
                raise InvalidInput("ranges must be > 0")
            radius, ratios = major, (semi / major, minor / major)
        self.radius = float(radius)
        self.max_samples = _count(max_samples, "max_samples")
        self.min_samples = _count(min_samples, "min_samples")
        self.octant = bool(octant)
        self.sectors = _count(sectors, "sectors")
        self.max_per_hole = _count(max_per_hole, "max_per_hole")
        self.min_sectors = _count(min_sectors, "min_sectors")
        self.max_empty_sectors = _count(max_empty_sectors, "max_empty_sectors")
        self.min_holes = _count(min_holes, "min_holes")
        max_per_sector = _count(max_per_sector, "max_per_sector")
        if max_per_sector is not None and self.sectors is None and not self.octant:
            raise InvalidInput("max_per_sector needs octant or sectors")
        self.max_per_octant = max_per_sector if (self.octant and self.sectors is None) else None
        self._sector_cap = (max_per_sector if max_per_sector is not None else
                            -(-self.max_samples // max(self.sectors, 1))) if self.sectors is not None else None
        if rotation is None and ratios is None:
            self.rotation = self.ratios = None
            self.anisotropy = None
        else:
            self.rotation = tuple(rotation) if rotation is not None else (0.0, 0.0, 0.0)
            self.ratios = tuple(ratios) if ratios is not None else (1.0, 1.0)
            self.anisotropy = anisotropy(self.rotation, self.ratios)
        self._check()

    def _check(self):
        """crates/estimation/src/search.rs:214-264."""
        bad = lambda m: InvalidInput(m)  # noqa: E731
        if math.isnan(self.radius) or self.radius <= 0 or self.max_samples == 0 or \
                self.min_samples > self.max_samples:
            raise bad("need radius > 0 and 1 <= min_samples <= max_samples")
        if self.sectors is not None:
            if self.octant:
                raise bad("give octant or sectors, not both")
            if not (2 <= self.sectors <= 360) or self._sector_cap == 0:
                raise bad("sectors need 2 <= count <= 360 and max_per_sector >= 1")
            count = ring = self.sectors
        elif self.octant:
            count, ring = 8, 4
        else:
            count = ring = 0
        if self.max_per_octant == 0:
            raise bad("max_per_sector must be >= 1")
        if (self.min_sectors is not None or self.max_empty_sectors is not None) and not self.balances():
            raise bad("min_sectors and max_empty_sectors need octant or sectors")
        if self.min_sectors is not None and (self.min_sectors == 0 or self.min_sectors > count or
                                             self.min_sectors > self.max_samples):
            raise bad("min_sectors must be at least 1 and at most the number of sectors (8 octants) and "
                      "max_samples")
        if self.max_empty_sectors is not None and self.max_empty_sectors >= ring:
            raise bad("max_empty_sectors must be below the number of sectors (4 octants per half)")
        if self.min_holes is not None and (self.min_holes == 0 or self.min_holes > self.max_samples):
            raise bad("min_holes must be at least 1 and at most max_samples")

    def balances(self):
        return self.octant or self.sectors is not None

    @property
    def max_per_sector(self):
        """Cap per plane sector, or per octant when given with octant (crates/py/src/estimation.rs:599-606)."""
        return self._sector_cap if self.sectors is not None else self.max_per_octant

    @property
    def ranges(self):
        """(major, semi, minor) of the ellipsoid; None without an anisotropy of its own."""
        if self.anisotropy is None:
            return None
        return (self.radius, self.radius * self.anisotropy[4], self.radius * self.anisotropy[5])

    def _varied(self, factor, min_samples, max_samples, min_holes):
        """A copy with the ellipsoid scaled by `factor`, `min_samples` / `max_samples` in place of its own when
        given, and `min_holes` in place of its own, checked once all are set (crates/py/src/estimation.rs:276-307):
        plane sectors left at their default cap follow the new max_samples."""
        factor = float(factor)
        if not (math.isfinite(factor) and factor > 0):
            raise InvalidInput("factors must be finite and > 0")
        out = Search.__new__(Search)
        out.__dict__.update(self.__dict__)
        out.radius = self.radius * factor
        if min_samples is not None:
            out.min_samples = _count(min_samples, "min_samples")
        if max_samples is not None:
            out.max_samples = _count(max_samples, "max_samples")
            if self.sectors is not None and self._sector_cap == -(-self.max_samples // self.sectors):
                out._sector_cap = -(-out.max_samples // self.sectors)
        out.min_holes = _count(min_holes, "min_holes")
        out._check()
        return out

    def scaled(self, factor, min_samples=None, max_samples=None):
        """A pass with the ellipsoid scaled by `factor`, and `min_samples` / `max_samples` in place of its own
        (estimation.rs:276-307): plane sectors left at their default cap follow the new max_samples."""
        return self._varied(factor, min_samples, max_samples, self.min_holes)

    def _vary(self, factor, max_samples, min_holes):
        """A copy with the ellipsoid scaled by `factor`, and `max_samples` and `min_holes` (None: no hole rule)
        in place of its own; for calibrate_search (crates/py/src/estimation.rs:560-564)."""
        return self._varied(factor, None, max_samples, min_holes)

    @staticmethod
    def passes(base, factors=(1.0, 2.0, 3.0), *, min_samples=None, max_samples=None):
        """Passes of `base` with its ellipsoid widened by each factor, and one min_samples / max_samples per
        pass in place of the base's (crates/py/src/estimation.rs:511-557)."""
        factors = list(factors)
        if not factors:
            raise InvalidInput("passes need at least one factor")
        for given, what in ((min_samples, "min_samples"), (max_samples, "max_samples")):
            if given is not None and len(given) != len(factors):
                raise InvalidInput(f"{what}: expected {len(factors)} values, got {len(given)}")
        return [base.scaled(f, None if min_samples is None else min_samples[i],
                            None if max_samples is None else max_samples[i]) for i, f in enumerate(factors)]

    def to_json(self):
        """{"type": "Search", "format": 1, <the search's serde fields>} (crates/py/src/estimation.rs:401-412,
        crates/py/src/persist.rs:20-33)."""
        from .persist import envelope_of, search_json

        return envelope_of("Search", search_json(self))

    @staticmethod
    def from_json(text):
        """Reads to_json output; InvalidInput on another class's JSON or a newer format (persist.rs:35-51)."""
        from .persist import _open, search_from

        return search_from(_open("Search", text))

    def to_c(self):
        s = N.SearchC()
        none = -1
        s.min_samples, s.max_samples, s.radius = self.min_samples, self.max_samples, self.radius
        s.max_per_hole = none if self.max_per_hole is None else self.max_per_hole
        s.octant = 1 if self.octant else 0
        s.sectors = 0 if self.sectors is None else self.sectors
        s.max_per_sector = 0 if self._sector_cap is None else self._sector_cap
        s.max_per_octant = none if self.max_per_octant is None else self.max_per_octant
        s.min_sectors = none if self.min_sectors is None else self.min_sectors
        s.max_empty_sectors = none if self.max_empty_sectors is None else self.max_empty_sectors
        s.min_holes = none if self.min_holes is None else self.min_holes
        s.aniso = aniso_c(self.anisotropy)
        s.calibration = 1 if self.target_slope is not None else (2 if self.target_efficiency is not None else 0)
        s.calibration_target = (self.target_slope if self.target_slope is not None else
                                self.target_efficiency if self.target_efficiency is not None else 0.0)
        return s

    def calibrated(self):
        return self.target_slope is not None or self.target_efficiency is not None

    def __repr__(self):
        return (f"Search(radius={self.radius}, max_samples={self.max_samples}, min_samples={self.min_samples}, "
                f"octant={self.octant}, max_per_octant={self.max_per_octant}, anisotropy={self.anisotropy})")
