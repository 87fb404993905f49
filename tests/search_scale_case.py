"""The workload of the reference's search scale test (crates/estimation/tests/search_scale.rs:9-127): 504,100
composites of 5,041 drill holes, lattice targets among them, and the test's brute-force selection."""

import numpy as np

M1, M2 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)


def unit_hash(x):
    """search_scale.rs:9-13: a 64-bit mix of x to a double in [0, 1)."""
    x = np.asarray(x, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (x ^ (x >> np.uint64(30))) * M1
        x = (x ^ (x >> np.uint64(27))) * M2
    return ((x ^ (x >> np.uint64(31))) >> np.uint64(11)).astype(np.float64) / float(1 << 53)


def composites():
    """search_scale.rs:15-29: (locations (504100, 3), values, hole ids)."""
    h = np.repeat(np.arange(5041, dtype=np.uint64), 100)
    k = np.tile(np.arange(100, dtype=np.uint64), 5041)
    x0, y0 = (h % np.uint64(71)).astype(np.float64) * 30.0, (h // np.uint64(71)).astype(np.float64) * 30.0
    dx, dy = unit_hash(h) - 0.5, unit_hash(h + np.uint64(9999)) - 0.5
    d = k.astype(np.float64) * 4.0 + 2.0
    locs = np.column_stack([x0 + dx * 0.3 * d, y0 + dy * 0.3 * d, 400.0 - d])
    return locs, unit_hash(h * np.uint64(1000) + k), h.astype(np.int64)


def targets():
    """search_scale.rs:93-106: every 53rd of a 200 x 200 x 25 lattice of 5 m blocks and three targets that
    once lost a neighbour."""
    i = np.arange(0, 1_000_000, 53)
    t = np.column_stack([300.0 + (i % 200) * 5.0, 300.0 + (i // 200 % 200) * 5.0, 50.0 + (i // 40_000) * 5.0])
    return np.vstack([t, [[300.0, 1255.0, 205.0], [590.0, 820.0, 215.0], [575.0, 830.0, 210.0]]])


def brute(t, locs, holes, radius, max_samples, min_samples, max_per_hole=None, octant=False):
    """search_scale.rs:31-71: every sample by (squared distance, index) through the greedy rules of an
    isotropic search; None below min_samples."""
    d2 = (locs[:, 0] - t[0]) ** 2 + (locs[:, 1] - t[1]) ** 2 + (locs[:, 2] - t[2]) ** 2
    near = np.nonzero(d2 <= radius * radius)[0]
    order = near[np.lexsort((near, d2[near]))]
    cap = -(-max_samples // 8) if octant else None
    chosen, per_hole, per_octant = [], {}, [0] * 8
    for i in order:
        if len(chosen) >= max_samples:
            break
        h = int(holes[i])
        if max_per_hole is not None and per_hole.get(h, 0) >= max_per_hole:
            continue
        p = locs[i]
        o = (int(p[0] >= t[0]) << 2) | (int(p[1] >= t[1]) << 1) | int(p[2] >= t[2])
        if octant:
            if per_octant[o] >= cap:
                continue
            per_octant[o] += 1
        per_hole[h] = per_hole.get(h, 0) + 1
        chosen.append(int(i))
    return chosen if len(chosen) >= min_samples else None
