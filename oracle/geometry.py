"""Geometry and per-sublattice precompute of the reference, restated in numpy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``). This module is an independent restatement of
the reference's host-side precompute. Tests use it to check the product's C++ precompute (pair list,
packed species, shuffle windows, prefactors, scaled pair weights) and to feed the oracle's loop.

All arithmetic runs in the job's floating type ``T`` (numpy float32 / float64 scalars), in the
reference's operation order. Citations are reference paths relative to its repository root.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


def is_close(a, b, atol, rtol, T):
    """``core/helpers/numeric.h:11-14``: |a-b| <= atol + rtol*|b| evaluated in T."""
    a, b, atol, rtol = T(a), T(b), T(atol), T(rtol)
    return bool(abs(T(a - b)) <= T(atol + T(rtol * abs(b))))


def supercell(lattice, frac, species, a, b, c, T=np.float64):
    """``core/structure.h:335-366``.

    The inverse of the diagonal scale matrix follows Eigen's 3x3 cofactor inverse: each diagonal
    entry is the cofactor times 1/det.
    """
    lattice = np.asarray(lattice, dtype=T)
    frac = np.asarray(frac, dtype=T)
    if a * b * c == 0:
        raise ValueError("There must be at least one copy in each direction")
    da, db, dc = T(a), T(b), T(c)
    det = T(T(db * dc) * da)
    invdet = T(T(1) / det)
    inv = [T(T(db * dc) * invdet), T(T(da * dc) * invdet), T(T(da * db) * invdet)]
    n = frac.shape[0]
    scaled = np.empty_like(frac)
    for k in range(3):
        scaled[:, k] = frac[:, k] * inv[k]
    coords = np.empty((n * a * b * c, 3), dtype=T)
    out_species = []
    idx = 0
    for i in range(a):
        for j in range(b):
            for k in range(c):
                tr = np.array([T(i) * inv[0], T(j) * inv[1], T(k) * inv[2]], dtype=T)
                for s in range(n):
                    coords[idx] = tr + scaled[s]
                    out_species.append(int(species[s]))
                    idx += 1
    new_lattice = lattice.copy()
    for r in range(3):
        new_lattice[r, 0] = lattice[r, 0] * da
        new_lattice[r, 1] = lattice[r, 1] * db
        new_lattice[r, 2] = lattice[r, 2] * dc
    return new_lattice, coords, out_species


def distance_matrix(lattice, frac, T=np.float64):
    """``core/structure.h:35-69`` — minimum distance over the 27 images (-1, 0, 1)^3."""
    lattice = np.asarray(lattice, dtype=T)
    frac = np.asarray(frac, dtype=T)
    n = frac.shape[0]
    cart = np.empty_like(frac)
    for i in range(n):
        for j in range(3):
            # coefficient-wise inner product of three terms, summed x0 + (x1 + x2)
            x0 = T(frac[i, 0] * lattice[0, j])
            x1 = T(frac[i, 1] * lattice[1, j])
            x2 = T(frac[i, 2] * lattice[2, j])
            cart[i, j] = T(x0 + T(x1 + x2))
    la, lb, lc = lattice[0], lattice[1], lattice[2]
    shifts = []
    for u in (-1, 0, 1):
        for v in (-1, 0, 1):
            for w in (-1, 0, 1):
                shifts.append(((T(u) * la + T(v) * lb) + T(w) * lc).astype(T))
    shifts = np.array(shifts, dtype=T)  # (27, 3)
    d = np.full((n, n), np.finfo(T).max, dtype=T)
    for i in range(n):
        p1 = cart[i]
        for j in range(i, n):
            diff = (p1[None, :] - (shifts + cart[j][None, :])).astype(T)
            sq = diff * diff
            norms = np.sqrt((sq[:, 0] + (sq[:, 1] + sq[:, 2])).astype(T)).astype(T)
            m = norms.min()
            d[i, j] = m
            d[j, i] = m
    return d


def shell_matrix(dmat, dists, atol, rtol, T=np.float64):
    """``core/structure.h:71-100`` — shell index per pair, 0 on the diagonal."""
    dmat = np.asarray(dmat, dtype=T)
    dists = [T(x) for x in dists]
    n = dmat.shape[0]

    def find_shell(d):
        if d < 0:
            raise ValueError("Invalid distance matrix input")
        if is_close(d, 0.0, atol, rtol, T):
            return 0
        for i in range(len(dists) - 1):
            lb, up = dists[i], dists[i + 1]
            if (is_close(d, lb, atol, rtol, T) or d > lb) and (is_close(d, up, atol, rtol, T) or up > d):
                return i + 1
        return len(dists)

    sm = np.zeros((n, n), dtype=np.int64)
    cache = {}
    for i in range(n):
        for j in range(i + 1, n):
            d = dmat[i, j]
            key = float(d)
            if key not in cache:
                cache[key] = find_shell(d)
            sm[i, j] = sm[j, i] = cache[key]
    return sm


def distances_naive(dmat, atol, rtol, T=np.float64):
    """``core/structure.h:195-207`` — unique sorted distances, near-equal neighbours averaged."""
    vals = sorted(set(float(x) for x in np.asarray(dmat, dtype=T).reshape(-1)))
    vec = [T(0)]
    for v in vals:
        dist = T(v)
        if is_close(vec[-1], dist, atol, rtol, T):
            vec[-1] = T(0.5 * float(T(dist + vec[-1])))
        else:
            vec.append(dist)
    return vec


def distances_histogram(dmat, bin_width, peak_isolation, T=np.float64):
    """``core/structure.h:209-258`` — shell radii from isolated histogram peaks."""
    flat = [T(x) for x in np.asarray(dmat, dtype=T).reshape(-1, order="F")]
    distances = sorted(d for d in flat if d > 0.0 and not is_close(d, 0.0, 1e-5, 1e-3, T))
    bin_width = T(bin_width)
    mn, mx = distances[0], distances[-1]
    num_edges = int(T(T(mx - mn) / bin_width)) + 2
    edges = [T(mn + T(T(i) * bin_width)) for i in range(num_edges)]
    if len(edges) < 10:
        raise ValueError("Not enough edges to create a histogram, please increase the bin width")
    freqs = {0: []}
    index = 0
    b = 0
    while index < len(distances) and b < num_edges - 1:
        lower, upper, value = edges[b], edges[b + 1], distances[index]
        if lower <= value < upper:
            freqs[b].append(value)
            index += 1
        else:
            b += 1
            freqs[b] = []
    shells = []
    pi = float(T(peak_isolation))
    for i in range(num_edges + 1):
        prev, f, nxt = freqs.get(i - 1, []), freqs.get(i, []), freqs.get(i + 1, [])
        threshold = int((1.0 - pi) * float(T(len(f))))
        if threshold > len(prev) and threshold > len(nxt):
            shells.append(max(f))
    if shells[0] != 0.0 and not is_close(shells[0], 0.0, 1e-5, 1e-3, T):
        shells.insert(0, T(0))
    return shells


def make_index_mapping(values):
    """``core/helpers.h:93-107`` — sorted distinct values to dense indices (and back)."""
    uniq = sorted(set(int(v) for v in values))
    fwd = {v: i for i, v in enumerate(uniq)}
    rev = {i: v for i, v in enumerate(uniq)}
    return fwd, rev


def compute_prefactors(smat, weights, species, T=np.float64):
    """``core/structure.h:136-192``.

    The per-shell neighbour count is stored back into a ``counter<usize_t>`` (an integer map), so
    count/N is truncated to an integer before it becomes M_i.
    """
    if not weights:
        raise ValueError("no coordination shells selected")
    n = len(species)
    vals, counts = np.unique(np.asarray(smat).reshape(-1), return_counts=True)
    neighbors = {}
    for shell, cnt in zip(vals.tolist(), counts.tolist()):
        per = T(T(cnt) / T(n))
        neighbors[int(shell)] = int(per)  # truncation into size_t
    shell_rev = make_index_mapping(weights.keys())[1]
    conf_rev = make_index_mapping(species)[1]
    hist = {}
    for z in species:
        hist[int(z)] = hist.get(int(z), 0) + 1
    K = len(hist)
    S = len(weights)
    out = np.zeros((S, K, K), dtype=T)
    for s in range(S):
        nc = neighbors.get(shell_rev[s], 0)
        if nc > 0:
            M = T(nc)
            for a in range(K):
                xa = T(T(hist[conf_rev[a]]) / T(n))
                for b in range(a, K):
                    xb = T(T(hist[conf_rev[b]]) / T(n))
                    p = T(T(1.0) / T(T(T(M * xa) * xb) * T(n)))
                    out[s, a, b] = p
                    out[s, b, a] = p
    return out


def pairs(smat, weights):
    """``core/structure.h:434-451`` — (i, j, packed shell) for i < j whose shell has a weight."""
    fwd = make_index_mapping(weights.keys())[0]
    smat = np.asarray(smat)
    n = smat.shape[0]
    out = []
    for i in range(n):
        for j in range(i + 1, n):
            s = int(smat[i, j])
            if s in weights:
                out.append((i, j, fwd[s]))
    return np.array(out, dtype=np.uint32).reshape(-1, 3)


def scaled_pair_weights(pair_weights, weights, K, T=np.float64):
    """``core/optimization.h:17-33``."""
    w = np.array(pair_weights, dtype=T, copy=True)
    rev = make_index_mapping(weights.keys())[1]
    for s in range(len(weights)):
        ws = T(weights[rev[s]])
        for xi in range(K):
            for eta in range(xi, K):
                w[s, xi, eta] = T(w[s, xi, eta] * ws)
                if xi == eta:
                    continue
                w[s, eta, xi] = T(w[s, eta, xi] * ws)
    return w


def apply_composition(species, composition):
    """``core/structure.h:390-396`` — fill each sublattice's sorted sites, lowest Z first."""
    out = list(species)
    for sites, comp in composition:
        it = iter(sorted(sites))
        for z in sorted(comp):
            for _ in range(comp[z]):
                out[next(it)] = int(z)
    return out


def shuffling_bounds(n_sites, composition):
    """``core/optimization.h:35-72`` — sort sites by sublattice index and cut windows.

    The reference sorts with libstdc++ ``std::sort`` (not stable), which permutes sites with equal
    keys; the oracle library restates the step with the same call (``oracle.sort_by_sublattice``).
    """
    from . import sort_by_sublattice

    sl_of = []
    for site in range(n_sites):
        k = next((i for i, (sites, _) in enumerate(composition) if site in sites), len(composition))
        sl_of.append(k)
    return sort_by_sublattice(sl_of, len(composition))


def default_shell_weights(n_radii, T=np.float64):
    """``io/config/shell_weights.h:75-83`` — {i: 1/i} for i in [1, len(radii))."""
    return {i: T(T(1.0) / T(i)) for i in range(1, n_radii)}


@dataclass
class SublatticeData:
    n_sites: int
    species_packed: np.ndarray
    pairs: np.ndarray
    bounds: list
    prefactors: np.ndarray
    pair_weights: np.ndarray
    target: np.ndarray
    sort_order: list
    species_rev: dict
    shell_weights: dict
    radii: list = field(default_factory=list)


def prepare_interact(lattice, frac, species, composition, radii, weights, T=np.float64,
                     prefactors=None, pair_weights=None, target=None):
    """``core/optimization_config.h:59-141`` for sublattice mode "interact".

    ``species`` are the structure's atomic numbers after the supercell; ``composition`` is a list
    of (sites, {Z: count}). Arrays default like ``io/config/arrays.h:103-107,155-190``.
    """
    n = len(species)
    st_species = apply_composition(species, composition)
    dmat = distance_matrix(lattice, frac, T)
    eps = np.finfo(T).eps
    smat = shell_matrix(dmat, radii, eps, 1e-9, T)
    K = len(set(st_species))
    S = len(weights)
    if prefactors is None:
        prefactors = compute_prefactors(smat, weights, st_species, T)
    if pair_weights is None:
        pair_weights = np.stack([np.ones((K, K), dtype=T) - np.eye(K, dtype=T)] * S)
    if target is None:
        target = np.zeros((S, K, K), dtype=T)
    order, bounds = shuffling_bounds(n, composition)
    sorted_species = [st_species[i] for i in order]
    fwd, rev = make_index_mapping(sorted_species)
    packed = np.array([fwd[z] for z in sorted_species], dtype=np.uint8)
    # pairs of the sorted structure: permute the shell matrix instead of recomputing distances
    sm_sorted = smat[np.ix_(order, order)]
    pl = pairs(sm_sorted, weights)
    w = scaled_pair_weights(pair_weights, weights, K, T)
    return SublatticeData(n, packed, pl, bounds, np.asarray(prefactors, dtype=T), w,
                          np.asarray(target, dtype=T), order, rev, dict(weights), list(radii))


def prepare_split_sublattice(lattice, frac, species, composition, index, radii, weights,
                             T=np.float64, prefactors=None, pair_weights=None, target=None):
    """One sublattice of ``apply_composition_and_decompose`` (core/structure.h:406-411)."""
    st_species = apply_composition(species, composition)
    sites = sorted(composition[index][0])
    sub_frac = np.asarray(frac, dtype=T)[sites]
    sub_species = [st_species[i] for i in sites]
    dmat = distance_matrix(lattice, sub_frac, T)
    eps = np.finfo(T).eps
    smat = shell_matrix(dmat, radii, eps, 1e-9, T)
    K = len(set(sub_species))
    S = len(weights)
    if prefactors is None:
        prefactors = compute_prefactors(smat, weights, sub_species, T)
    if pair_weights is None:
        pair_weights = np.stack([np.ones((K, K), dtype=T) - np.eye(K, dtype=T)] * S)
    if target is None:
        target = np.zeros((S, K, K), dtype=T)
    fwd, rev = make_index_mapping(sub_species)
    packed = np.array([fwd[z] for z in sub_species], dtype=np.uint8)
    pl = pairs(smat, weights)
    w = scaled_pair_weights(pair_weights, weights, K, T)
    n = len(sites)
    return SublatticeData(n, packed, pl, [(0, n)], np.asarray(prefactors, dtype=T), w,
                          np.asarray(target, dtype=T), list(range(n)), rev, dict(weights), list(radii))


def fcc(a):
    """Conventional fcc cell (4 sites)."""
    return (np.eye(3) * a, np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]))


def bcc(a):
    """Conventional bcc cell (2 sites)."""
    return (np.eye(3) * a, np.array([[0, 0, 0], [0.5, 0.5, 0.5]]))


def rocksalt(a):
    """Conventional rock-salt cell (8 sites: 4 cations then 4 anions)."""
    cat = [[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]
    an = [[0.5, 0, 0], [0, 0.5, 0], [0, 0, 0.5], [0.5, 0.5, 0.5]]
    return (np.eye(3) * a, np.array(cat + an))


def coordination_numbers(prefactors, n_sites):
    """Inverse of a one-species prefactor cube: 1/f/N per shell (tests/test_structure.cpp:219-221)."""
    return [int((1.0 / float(p)) / float(n_sites)) for p in np.asarray(prefactors).reshape(-1)]


__all__ = [name for name in dir() if not name.startswith("_") and name not in ("math", "np", "dataclass", "field")]
