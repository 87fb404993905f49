"""ORACLE — test infrastructure only.

ctypes access to the C++ restatement of the reference kriging path
(oracle/boitata_oracle.cpp, built into oracle/_build/liboracle.so by
oracle/Makefile). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use it, as the reference results are compared with; the product
never does.

Parameter objects are read by attribute (nugget, structures, anisotropy for
a variogram; radius, counts, octant, anisotropy for a search), so the
product's Variogram/Search objects and plain namespaces both work.
"""

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
MODELS = {"spherical": 0, "exponential": 1, "gaussian": 2, "cubic": 3, "pentaspherical": 4, "circular": 5,
          "sinehole": 6, "matern": 7, "power": 8}
KINDS = {"ordinary": 0, "simple": 1, "indicator": 2}
OK, SEARCH_FAILED, SINGULAR, INSUFFICIENT, INVALID, NONE = 0, 1, 2, 3, 4, -1


class Aniso(ctypes.Structure):
    _fields_ = [("on", ctypes.c_int32), ("azimuth", ctypes.c_double), ("dip", ctypes.c_double),
                ("rake", ctypes.c_double), ("major", ctypes.c_double), ("semi", ctypes.c_double),
                ("minor", ctypes.c_double)]


class Struct(ctypes.Structure):
    _fields_ = [("model", ctypes.c_int32), ("param", ctypes.c_double), ("sill", ctypes.c_double),
                ("range", ctypes.c_double)]


class Vario(ctypes.Structure):
    _fields_ = [("nugget", ctypes.c_double), ("nstruct", ctypes.c_int32), ("s", Struct * 4), ("aniso", Aniso)]


class Srch(ctypes.Structure):
    _fields_ = [("min_samples", ctypes.c_int64), ("max_samples", ctypes.c_int64), ("radius", ctypes.c_double),
                ("max_per_hole", ctypes.c_int64), ("octant", ctypes.c_int64), ("sectors", ctypes.c_int64),
                ("max_per_sector", ctypes.c_int64), ("max_per_octant", ctypes.c_int64),
                ("min_sectors", ctypes.c_int64), ("max_empty_sectors", ctypes.c_int64),
                ("min_holes", ctypes.c_int64), ("aniso", Aniso), ("calibration", ctypes.c_int64),
                ("calibration_target", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("variance", ctypes.c_double), ("lagrange", ctypes.c_double),
                ("support", ctypes.c_double), ("n_used", ctypes.c_int64), ("status", ctypes.c_int32)]


_lib = None
P = ctypes.c_void_p


def build():
    """Compiles the oracle (g++, no FMA contraction) when its source is newer."""
    src = os.path.join(HERE, "boitata_oracle.cpp")
    if os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src):
        return LIB_PATH
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "orc_num_threads": (ctypes.c_int, []),
            "orc_rotation_matrix": (None, [ctypes.c_double] * 3 + [P]),
            "orc_block_frame": (None, [ctypes.c_double] * 3 + [P]),
            "orc_aniso_matrix": (None, [ctypes.POINTER(Aniso), P]),
            "orc_shape": (ctypes.c_double, [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
            "orc_shape_d1": (ctypes.c_double, [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
            "orc_cov": (ctypes.c_double, [ctypes.POINTER(Vario), ctypes.c_double]),
            "orc_cov_points": (ctypes.c_double, [ctypes.POINTER(Vario), P, P]),
            "orc_check_search": (ctypes.c_int32, [ctypes.POINTER(Srch)]),
            "orc_krige": (ctypes.c_int32, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, P, ctypes.c_int64, P, P,
                                           P, ctypes.POINTER(Vario), ctypes.POINTER(Result), P]),
            "orc_grid_visit": (ctypes.c_int64, [ctypes.c_int64, P, P, ctypes.c_double, P, P, ctypes.c_int64]),
            "orc_tree_new": (P, [ctypes.c_int64, P, P, ctypes.POINTER(Srch), ctypes.POINTER(Vario)]),
            "orc_tree_free": (None, [P]),
            "orc_tree_neighbors": (ctypes.c_int32, [P, P, ctypes.c_int64, P, P]),
            "orc_scan_neighbors": (ctypes.c_int32, [ctypes.c_int64, P, P, ctypes.POINTER(Srch),
                                                    ctypes.POINTER(Vario), P, P, P]),
            "orc_estimate_many": (ctypes.c_int32, [ctypes.c_int64, P, ctypes.c_int32, ctypes.c_int64, P, P, P, P,
                                                   ctypes.POINTER(Srch), ctypes.POINTER(Vario), ctypes.c_int32,
                                                   ctypes.c_double, ctypes.c_int32, P, P, P, P, P]),
            "orc_k_fold": (ctypes.c_int32, [ctypes.c_int64, ctypes.c_int64, P, P, P, P, P, ctypes.POINTER(Srch),
                                            ctypes.POINTER(Vario), ctypes.c_int32, ctypes.c_double, P]),
            "orc_centroids": (None, [P, P, P, P, ctypes.c_int64, ctypes.c_int64, P]),
            "orc_sgs": (ctypes.c_int64, [ctypes.c_int64, P, P, P, ctypes.c_int64, P, P, ctypes.POINTER(Srch),
                                         ctypes.POINTER(Vario), P, P]),
            "orc_prefix_quality": (None, [ctypes.c_int64, P, P, P, ctypes.POINTER(Vario), ctypes.c_int32,
                                          ctypes.c_double, P, P, P]),
            "orc_krige_lists": (ctypes.c_int32, [ctypes.c_int64, P, ctypes.c_int64, P, P, P, P, ctypes.c_int64,
                                                 ctypes.POINTER(Vario), ctypes.c_int32, ctypes.c_double,
                                                 ctypes.c_int32, P]),
            "orc_block_offsets": (None, [P, P, P, P]),
            "orc_block_krige": (ctypes.c_int32, [P, ctypes.c_int64, P, ctypes.c_int64, P, P, P,
                                                 ctypes.POINTER(Vario), ctypes.POINTER(Result), P]),
            "orc_estimate_block": (ctypes.c_int32, [ctypes.c_int64, P, ctypes.c_int64, P, P, P, P,
                                                    ctypes.POINTER(Srch), ctypes.POINTER(Vario), ctypes.c_int64, P,
                                                    ctypes.c_int32, P]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def aniso(a):
    out = Aniso()
    if a is not None:
        out.on = 1
        out.azimuth, out.dip, out.rake, out.major, out.semi, out.minor = (float(v) for v in a)
    return out


def variogram(vg):
    v = Vario()
    v.nugget = vg.nugget
    v.nstruct = len(vg.structures)
    for k, s in enumerate(vg.structures):
        code = MODELS[s.model]
        param = s.order if s.model == "matern" else (s.exponent if s.model == "power" else 0.0)
        v.s[k].model, v.s[k].param, v.s[k].sill, v.s[k].range = code, param or 0.0, s.sill, s.range
    v.aniso = aniso(vg.anisotropy)
    return v


def search(s):
    c = Srch()
    none = lambda x: -1 if x is None else int(x)  # noqa: E731
    c.min_samples, c.max_samples, c.radius = s.min_samples, s.max_samples, s.radius
    c.max_per_hole = none(getattr(s, "max_per_hole", None))
    c.octant = int(bool(s.octant))
    c.sectors = getattr(s, "sectors", None) or 0
    c.max_per_sector = getattr(s, "max_per_sector", None) or 0
    c.max_per_octant = none(getattr(s, "max_per_octant", None))
    c.min_sectors = none(getattr(s, "min_sectors", None))
    c.max_empty_sectors = none(getattr(s, "max_empty_sectors", None))
    c.min_holes = none(getattr(s, "min_holes", None))
    c.aniso = aniso(s.anisotropy)
    slope, eff = getattr(s, "target_slope", None), getattr(s, "target_efficiency", None)
    c.calibration = 1 if slope is not None else (2 if eff is not None else 0)
    c.calibration_target = slope if slope is not None else (eff if eff is not None else 0.0)
    return c


def _xyz(a):
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 2 and a.shape[1] == 2:
        a = np.column_stack([a, np.zeros(len(a))])
    return np.ascontiguousarray(a)


def rotation_matrix(az, dip, rake):
    out = np.empty(9)
    lib().orc_rotation_matrix(az, dip, rake, out.ctypes.data)
    return out.reshape(3, 3)


def block_frame(az, dip, rake):
    out = np.empty(9)
    lib().orc_block_frame(az, dip, rake, out.ctypes.data)
    return out.reshape(3, 3)


def aniso_matrix(a):
    out = np.empty(9)
    x = aniso(a)
    lib().orc_aniso_matrix(ctypes.byref(x), out.ctypes.data)
    return out.reshape(3, 3)


def shape(model, h, rng, param=0.0):
    return lib().orc_shape(MODELS[model], param, h, rng)


def shape_d1(model, h, rng, param=0.0):
    return lib().orc_shape_d1(MODELS[model], param, h, rng)


def cov(vg, h):
    v = variogram(vg)
    return lib().orc_cov(ctypes.byref(v), h)


def cov_points(vg, p, q):
    v = variogram(vg)
    p = np.ascontiguousarray(p, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_cov_points(ctypes.byref(v), p.ctypes.data, q.ctypes.data)


def check_search(s):
    c = search(s)
    return bool(lib().orc_check_search(ctypes.byref(c)))


def krige(kind, target, xyz, values, vg, *, kparam=0.0, err=None, which="krige"):
    """(status, {value, variance, lagrange, support, n_used}, weights) of one system (krige.rs:83-95);
    which = 'krige' (guard + kernel + LU), 'kernel' (kernel.rs only) or 'lu' (krige_lu)."""
    xyz = _xyz(xyz)
    n = len(xyz)
    v = np.ascontiguousarray(values, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    t = np.ascontiguousarray(target, dtype=np.float64)
    if t.shape == (2,):
        t = np.array([t[0], t[1], 0.0])
    w = np.zeros(max(n, 1))
    r = Result()
    vv = variogram(vg)
    st = lib().orc_krige({"krige": 0, "kernel": 1, "lu": 2}[which], KINDS[kind], kparam, t.ctypes.data, n,
                         xyz.ctypes.data, v.ctypes.data, _ptr(e), ctypes.byref(vv), ctypes.byref(r), w.ctypes.data)
    out = dict(value=r.value, variance=r.variance, lagrange=r.lagrange, support=r.support, n_used=r.n_used)
    return st, out, w[:n]


def grid_visit(pts, q, radius2, stop_after=0):
    """(d2 bits, index) stream of search/grid.rs `nearest` over pts."""
    pts = _xyz(pts)
    q = np.ascontiguousarray(q, dtype=np.float64)
    idx = np.empty(len(pts), dtype=np.int64)
    bits = np.empty(len(pts), dtype=np.uint64)
    k = lib().orc_grid_visit(len(pts), pts.ctypes.data, q.ctypes.data, radius2, idx.ctypes.data, bits.ctypes.data,
                             stop_after)
    return list(zip(bits[:k].tolist(), idx[:k].tolist()))


class Tree:
    """SearchTree (search.rs:692-1006) over samples, for neighbour queries."""

    def __init__(self, xyz, s, vg=None, holes=None):
        self._xyz = _xyz(xyz)
        self._holes = None if holes is None else np.ascontiguousarray(holes, dtype=np.int64)
        self._s, self._v = search(s), (None if vg is None else variogram(vg))
        self._max = int(s.max_samples)
        self._h = lib().orc_tree_new(len(self._xyz), self._xyz.ctypes.data, _ptr(self._holes), ctypes.byref(self._s),
                                     None if self._v is None else ctypes.byref(self._v))

    def neighbors(self, target, left_out=-1):
        """(ok, indices in selection order)."""
        t = np.ascontiguousarray(target, dtype=np.float64)
        out = np.empty(min(self._max, len(self._xyz)) + 1, dtype=np.int64)
        n = ctypes.c_int64(0)
        ok = lib().orc_tree_neighbors(self._h, t.ctypes.data, left_out, out.ctypes.data, ctypes.byref(n))
        return bool(ok), out[: n.value].tolist()

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_tree_free(self._h)
            self._h = None


def scan_neighbors(target, xyz, s, vg=None, holes=None):
    """neighbors_in by linear scan (search.rs:647-687): (ok, indices)."""
    xyz = _xyz(xyz)
    h = None if holes is None else np.ascontiguousarray(holes, dtype=np.int64)
    cs, cv = search(s), (None if vg is None else variogram(vg))
    t = np.ascontiguousarray(target, dtype=np.float64)
    out = np.empty(len(xyz) + 1, dtype=np.int64)
    n = ctypes.c_int64(0)
    ok = lib().orc_scan_neighbors(len(xyz), xyz.ctypes.data, _ptr(h), ctypes.byref(cs),
                                  None if cv is None else ctypes.byref(cv), t.ctypes.data, out.ctypes.data,
                                  ctypes.byref(n))
    return bool(ok), out[: n.value].tolist()


def prefix_quality(target, xyz, vg, *, ordinary=True, support=None, err=None):
    """(slope, efficiency, ok) of kriging `target` from each leading part of `xyz`
    (kriging_algebra.rs:336-395); ok False where the reference gives None."""
    xyz = _xyz(xyz)
    n = len(xyz)
    t = np.ascontiguousarray(target, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    sl, ef, ok = np.empty(n), np.empty(n), np.empty(n, dtype=np.int32)
    sv = vg.total_sill() if support is None else float(support)
    lib().orc_prefix_quality(n, xyz.ctypes.data, _ptr(e), t.ctypes.data, ctypes.byref(variogram(vg)),
                             1 if ordinary else 0, sv, sl.ctypes.data, ef.ctypes.data, ok.ctypes.data)
    return sl, ef, ok.astype(bool)


def sgs(xyz, scores, nodes, z, s, vg, *, holes=None):
    """Sequential simulation of `nodes` (in simulation order) from data `xyz` with normal `scores`
    (crates/simulation/src/sgs.rs:586-760): (node scores, how: 1 kriged, 2 marginal)."""
    xyz, nodes = _xyz(xyz), _xyz(nodes)
    sc = np.ascontiguousarray(scores, dtype=np.float64)
    zz = np.ascontiguousarray(z, dtype=np.float64)
    h = None if holes is None else np.ascontiguousarray(holes, dtype=np.int64)
    m = len(nodes)
    out, how = np.empty(m), np.zeros(m, dtype=np.int8)
    rc = lib().orc_sgs(len(xyz), xyz.ctypes.data, sc.ctypes.data, _ptr(h), m, nodes.ctypes.data, zz.ctypes.data,
                       ctypes.byref(search(s)), ctypes.byref(variogram(vg)), out.ctypes.data, how.ctypes.data)
    if rc < 0:
        raise ValueError(f"oracle: kriging failed at node {-1 - rc}")
    return out, how


def estimate_many(targets, xyz, values, s, vg, *, kind="ordinary", kparam=0.0, err=None, holes=None, loo=False,
                  threads=0, neighbors=True, diagnostics=False, domains=None, target_domains=None):
    """estimate_many / leave_one_out_at (batch.rs:15-38, 165-190) with krige of `kind`. With `diagnostics`,
    also the per-target columns of the diagnostics table that need the samples or weights
    (crates/py/src/estimation.rs:1046-1105): negative_weight_sum, mean_distance, n_holes, n_within and
    target_met (NaN without a calibration). With `domains` (the samples' codes) each target krigs from its
    own domain, `target_domains` (a code < 0: a domain without samples, not estimated); leave-one-out takes
    each sample's own."""
    xyz = _xyz(xyz)
    n = len(xyz)
    t = None if loo else _xyz(targets)
    m = n if loo else len(t)
    res = (Result * max(m, 1))()
    nbr = np.empty((m, int(s.max_samples)), dtype=np.int64) if neighbors else None
    v = np.ascontiguousarray(values, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    h = None if holes is None else np.ascontiguousarray(holes, dtype=np.int64)
    dg = np.empty((m, 5)) if diagnostics else None
    cs, cv = search(s), variogram(vg)
    sd = None if domains is None else np.ascontiguousarray(domains, dtype=np.int64)
    td = None if target_domains is None else np.ascontiguousarray(target_domains, dtype=np.int64)
    if sd is not None and not loo and td is None:
        raise ValueError("oracle: samples with domains need target domains")
    rc = lib().orc_estimate_many(m, _ptr(t), 1 if loo else 0, n, xyz.ctypes.data, v.ctypes.data, _ptr(e), _ptr(h),
                                 ctypes.byref(cs), ctypes.byref(cv), KINDS[kind], kparam, threads,
                                 ctypes.cast(res, P), _ptr(nbr), _ptr(dg), _ptr(sd), _ptr(td))
    if rc != 0:
        raise ValueError("oracle: invalid search parameters")
    arr = np.ctypeslib.as_array(ctypes.cast(res, ctypes.POINTER(ctypes.c_byte)), shape=(ctypes.sizeof(Result) * m,))
    rec = np.frombuffer(arr.tobytes(), dtype=np.dtype([("value", "f8"), ("variance", "f8"), ("lagrange", "f8"),
                                                        ("support", "f8"), ("n_used", "i8"), ("status", "i4"),
                                                        ("pad", "i4")]), count=m)
    out = {k: rec[k].copy() for k in ("value", "variance", "lagrange", "n_used", "status")}
    if neighbors:
        out["neighbors"] = nbr
    if diagnostics:
        out["support"] = rec["support"].copy()
        for j, key in enumerate(("negative_weight_sum", "mean_distance", "n_holes", "n_within", "target_met")):
            out[key] = dg[:, j].copy()
    return out


def k_fold(k, xyz, values, s, vg, *, kind="ordinary", kparam=0.0, err=None, holes=None, domains=None):
    """k_fold_at over every sample (batch.rs:197-243): {value, variance, lagrange, n_used, status}."""
    xyz = _xyz(xyz)
    n = len(xyz)
    v = np.ascontiguousarray(values, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    h = None if holes is None else np.ascontiguousarray(holes, dtype=np.int64)
    sd = None if domains is None else np.ascontiguousarray(domains, dtype=np.int64)
    res = (Result * max(n, 1))()
    rc = lib().orc_k_fold(int(k), n, xyz.ctypes.data, v.ctypes.data, _ptr(e), _ptr(h), _ptr(sd),
                          ctypes.byref(search(s)), ctypes.byref(variogram(vg)), KINDS[kind], kparam,
                          ctypes.cast(res, P))
    if rc != 0:
        raise ValueError("oracle: invalid search parameters or k")
    return _records(res, n)


def _records(res, m):
    arr = np.ctypeslib.as_array(ctypes.cast(res, ctypes.POINTER(ctypes.c_byte)), shape=(ctypes.sizeof(Result) * m,))
    rec = np.frombuffer(arr.tobytes(), dtype=np.dtype([("value", "f8"), ("variance", "f8"), ("lagrange", "f8"),
                                                        ("support", "f8"), ("n_used", "i8"), ("status", "i4"),
                                                        ("pad", "i4")]), count=m)
    return {k: rec[k].copy() for k in ("value", "variance", "lagrange", "n_used", "status")}


def krige_lists(targets, xyz, values, nbr, vg, *, kind="ordinary", kparam=0.0, err=None, skip_coincident=True):
    """krige of each target from its given neighbour list (m x k, -1 padded)."""
    xyz, t = _xyz(xyz), _xyz(targets)
    nbr = np.ascontiguousarray(nbr, dtype=np.int64)
    m, k = nbr.shape
    v = np.ascontiguousarray(values, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    res = (Result * max(m, 1))()
    cv = variogram(vg)
    lib().orc_krige_lists(m, t.ctypes.data, len(xyz), xyz.ctypes.data, v.ctypes.data, _ptr(e), nbr.ctypes.data, k,
                          ctypes.byref(cv), KINDS[kind], kparam, 1 if skip_coincident else 0, ctypes.cast(res, P))
    return _records(res, m)


def centroids(origin, size, count, rotation, first=0, m=None):
    """Geometry::centroid of cells first..first+m (block_model.rs:76-86)."""
    o = np.ascontiguousarray(origin, dtype=np.float64)
    s = np.ascontiguousarray(size, dtype=np.float64)
    c = np.ascontiguousarray(count, dtype=np.int64)
    r = np.ascontiguousarray(rotation, dtype=np.float64)
    if m is None:
        m = int(np.prod(c)) - first
    out = np.empty((m, 3))
    lib().orc_centroids(o.ctypes.data, s.ctypes.data, c.ctypes.data, r.ctypes.data, first, m, out.ctypes.data)
    return out


def num_threads():
    return lib().orc_num_threads()


def block_offsets(size, disc, rotation=(0.0, 0.0, 0.0)):
    """Discretization::offsets (block.rs:61-72): (nx ny nz, 3) points of a block of `size` centred at the
    origin, turned by `rotation`."""
    sz = np.ascontiguousarray(size, dtype=np.float64)
    nd = np.ascontiguousarray(disc, dtype=np.int64)
    r = np.ascontiguousarray(rotation, dtype=np.float64)
    out = np.empty((int(np.prod(nd)), 3))
    lib().orc_block_offsets(sz.ctypes.data, nd.ctypes.data, r.ctypes.data, out.ctypes.data)
    return out


def block_krige(target, offsets, xyz, values, vg, *, err=None):
    """block_krige_points (block.rs:120-198, ordinary) of one block centred at `target`: (status,
    {value, variance, lagrange, support, n_used}, weights)."""
    xyz = _xyz(xyz)
    n = len(xyz)
    t = np.ascontiguousarray(target, dtype=np.float64)
    off = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1, 3)
    v = np.ascontiguousarray(values, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    r = Result()
    w = np.zeros(max(n, 1))
    st = lib().orc_block_krige(t.ctypes.data, len(off), off.ctypes.data, n, xyz.ctypes.data, v.ctypes.data,
                               _ptr(e), ctypes.byref(variogram(vg)), ctypes.byref(r), w.ctypes.data)
    out = dict(value=r.value, variance=r.variance, lagrange=r.lagrange, support=r.support, n_used=r.n_used)
    return int(st), out, w[:n]


def estimate_block(targets, xyz, values, s, vg, offsets, *, err=None, holes=None, threads=0):
    """Block kriging of block centres `targets` (search at the centre, then block_krige_points over centre +
    offsets), as crates/py/src/estimation.rs:775-784 runs Method::Block."""
    xyz, t = _xyz(xyz), _xyz(targets)
    off = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1, 3)
    m = len(t)
    res = (Result * max(m, 1))()
    v = np.ascontiguousarray(values, dtype=np.float64)
    e = None if err is None else np.ascontiguousarray(err, dtype=np.float64)
    h = None if holes is None else np.ascontiguousarray(holes, dtype=np.int64)
    rc = lib().orc_estimate_block(m, t.ctypes.data, len(xyz), xyz.ctypes.data, v.ctypes.data, _ptr(e), _ptr(h),
                                  ctypes.byref(search(s)), ctypes.byref(variogram(vg)), len(off), off.ctypes.data,
                                  threads, ctypes.cast(res, P))
    if rc != 0:
        raise ValueError("oracle: invalid search parameters")
    return _records(res, m)
