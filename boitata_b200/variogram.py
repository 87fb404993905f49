"""Variogram parameters, as the reference's Python classes take them.

Mirrors crates/py/src/variogram.rs (Structure :179-256, Variogram :270-361,
`anisotropy` :164-177, `model` :28-51) over the core model of
crates/variogram/src/{model,composite,aniso}.rs: a nugget plus nested
structures sharing ONE anisotropy, whose major range is 1 so `ratios` are
semi/major and minor/major and each structure's range is along the major
axis.
"""

import math

from . import _native as N
from .errors import InvalidInput


def model_code(name, order=None, exponent=None):
    """Canonical model name and (code, param) for `name` (variogram.rs:28-51)."""
    key = str(name).lower().replace("-", "").replace("_", "").replace(" ", "")
    if key == "hole":
        key = "sinehole"
    if key not in N.MODELS:
        raise InvalidInput(f"unknown model {key!r}")
    if key == "matern":
        return key, N.MODELS[key], 1.5 if order is None else float(order)
    if key == "power":
        return key, N.MODELS[key], 1.0 if exponent is None else float(exponent)
    return key, N.MODELS[key], 0.0


class Structure:
    """One nested structure: `sill` is the partial sill, `range` the range along the major axis."""

    def __init__(self, model, sill, range, *, order=None, exponent=None):
        self.model, self._code, self._param = model_code(model, order, exponent)
        self.sill, self.range = float(sill), float(range)
        # crates/variogram/src/model.rs:47-59
        if not (self.sill >= 0 and math.isfinite(self.sill) and self.range > 0 and math.isfinite(self.range)):
            raise InvalidInput("structure sill must be finite and >= 0, range finite and > 0")

    @property
    def order(self):
        return self._param if self.model == "matern" else None

    @property
    def exponent(self):
        return self._param if self.model == "power" else None

    def to_json(self):
        """{"type": "Structure", "format": 1, "model": ..., "sill": ..., "range": ...} (variogram.rs:196-208)."""
        from .persist import envelope_of, variogram_json

        return envelope_of("Structure", variogram_json(Variogram([self]))["structures"][0])

    @staticmethod
    def from_json(text):
        from .persist import _open, variogram_from

        d = _open("Structure", text)
        return variogram_from({"nugget": 0.0, "structures": [d], "anisotropy": None}).structures[0]

    def __repr__(self):
        return f"Structure({self.model!r}, {self.sill}, {self.range})"


def anisotropy(rotation, ratios):
    """None for no anisotropy, else (azimuth, dip, rake, 1, semi, minor) (variogram.rs:164-177)."""
    rotation = tuple(float(v) for v in rotation)
    ratios = tuple(float(v) for v in ratios)
    if len(rotation) != 3 or len(ratios) != 2:
        raise InvalidInput("rotation needs (azimuth, dip, rake) and ratios (semi/major, minor/major)")
    if rotation == (0.0, 0.0, 0.0) and ratios == (1.0, 1.0):
        return None
    semi, minor = ratios
    # crates/variogram/src/aniso.rs:29-47
    if not all(r > 0 and math.isfinite(r) for r in (semi, minor)):
        raise InvalidInput("all ranges must be finite and > 0")
    if not all(math.isfinite(a) for a in rotation):
        raise InvalidInput("azimuth, dip and rake must be finite")
    return (*rotation, 1.0, semi, minor)


def aniso_c(a):
    out = N.Aniso()
    if a is not None:
        out.on = 1
        out.azimuth, out.dip, out.rake, out.major, out.semi, out.minor = a
    return out


class Variogram:
    """Nugget plus nested structures sharing one anisotropy (crates/py/src/variogram.rs:270-361)."""

    def __init__(self, structures, *, nugget=0.0, rotation=(0.0, 0.0, 0.0), ratios=(1.0, 1.0)):
        nugget = float(nugget)
        if not (nugget >= 0 and math.isfinite(nugget)):
            raise InvalidInput("nugget must be finite and >= 0")
        out = []
        for s in structures:
            if isinstance(s, Structure):
                out.append(s)
            else:
                try:
                    name, sill, rng = s
                except (TypeError, ValueError):
                    raise InvalidInput("structures are Structure or (model, sill, range) tuples") from None
                out.append(Structure(name, sill, rng))
        if len(out) > 4:
            raise InvalidInput("at most 4 nested structures")
        self.nugget = nugget
        self.structures = out
        self.rotation = tuple(float(v) for v in rotation)
        self.ratios = tuple(float(v) for v in ratios)
        self.anisotropy = anisotropy(self.rotation, self.ratios)

    def total_sill(self):
        """C(0) = nugget + sum of partial sills (composite.rs:50-52)."""
        return self.nugget + sum(s.sill for s in self.structures)

    def is_stationary(self):
        return all(s.model != "power" for s in self.structures)

    def to_c(self):
        v = N.VariogramC()
        v.nugget = self.nugget
        v.nstruct = len(self.structures)
        for k, s in enumerate(self.structures):
            v.s[k].model, v.s[k].param, v.s[k].sill, v.s[k].range = s._code, s._param, s.sill, s.range
        v.aniso = aniso_c(self.anisotropy)
        return v

    def with_params(self, nugget=None, sills=None, ranges=None, rotation=None, ratios=None):
        """A copy with some parameters replaced (for gradients and fitting)."""
        st = [Structure(s.model, sills[k] if sills is not None else s.sill,
                        ranges[k] if ranges is not None else s.range,
                        order=s.order, exponent=s.exponent) for k, s in enumerate(self.structures)]
        return Variogram(st, nugget=self.nugget if nugget is None else nugget,
                         rotation=self.rotation if rotation is None else rotation,
                         ratios=self.ratios if ratios is None else ratios)

    def to_json(self):
        """{"type": "Variogram", "format": 1, "nugget": ..., "structures": [...], "anisotropy": ...}
        (variogram.rs:569-579, composite.rs:12-18)."""
        from .persist import envelope_of, variogram_json

        return envelope_of("Variogram", variogram_json(self))

    @staticmethod
    def from_json(text):
        """Reads to_json output; InvalidInput on another class's JSON or a newer format."""
        from .persist import _open, variogram_from

        return variogram_from(_open("Variogram", text))

    def __repr__(self):
        return (f"Variogram({self.structures!r}, nugget={self.nugget}, rotation={self.rotation}, "
                f"ratios={self.ratios})")


__all__ = ["Structure", "Variogram", "anisotropy"]
