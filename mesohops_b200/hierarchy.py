"""Auxiliary hierarchy: generation, ordering and connection tables.

Aux vectors are rows of an integer count matrix [n_hier, n_mode].  Their order
is the reference's: basis/hops_aux.py:171-201,460-480 sorts by an id string that
lists each mode index (zero-padded to a fixed width) once per unit of depth,
shorter strings first and then lexicographically -- i.e. by total depth, then
lexicographically by the sorted tuple of modes.  For a full triangular
hierarchy that is the generation order of hops_hierarchy.py:340-368.

Instead of string ids this module ranks each aux exactly: the sorted mode
tuple c_0 <= ... <= c_{k-1} maps to the strictly increasing b_i = c_i + i in
[0, n), n = M + k - 1, whose lexicographic rank among the C(n, k)
combinations is sum_i C(n-1-b_{i-1}, k-i) - C(n-b_i, k-i) (b_{-1} = -1).
Adding the number of aux of depth < k gives a global key whose order equals
the reference order, so any aux subset is sorted, and neighbours are found,
with integer arithmetic (searchsorted) instead of string manipulation.  Where
the ranks exceed int64 (e.g. 500 modes to depth 10) the sort keys are
fixed-width byte strings (depth, then the sorted mode tuple, big-endian) with
the same order and equality.
"""
from __future__ import annotations

from math import comb

import numpy as np

from .exceptions import AuxError, UnsupportedRequest


def _binom_table(nmax, kmax):
    t = np.zeros((nmax + 1, kmax + 1), dtype=object)
    for n in range(nmax + 1):
        for k in range(kmax + 1):
            t[n, k] = comb(n, k)
    return t


class AuxKeyer:
    """Exact global keys of aux vectors for n_mode modes and depth <= maxhier."""

    def __init__(self, n_mode, maxhier):
        self.M = int(n_mode)
        self.D = int(maxhier)
        total = comb(self.M + self.D, self.D)  # aux of depth <= D
        self.use_int64 = total < (1 << 62)
        # offsets[k] = number of aux with depth < k = C(M + k - 1, k - 1)
        self.offsets = [0] + [comb(self.M + k - 1, k - 1) for k in range(1, self.D + 2)]
        nmax = self.M + self.D
        self.binom = _binom_table(nmax + 1, self.D + 1)
        if self.use_int64:
            self.binom64 = self.binom.astype(np.int64)

    def keys_from_counts(self, counts):
        """Global keys of aux given as a count matrix [N, M] (any int dtype)."""
        counts = np.asarray(counts)
        N = counts.shape[0]
        depth = counts.sum(axis=1).astype(np.int64)
        if depth.size and depth.max() > self.D:
            raise AuxError("aux deeper than MAXHIER")
        if self.use_int64:
            return self._keys_int64(counts, depth)
        keys = np.zeros(N, dtype=object)
        for k in np.unique(depth):
            idx = np.nonzero(depth == k)[0]
            if k == 0:
                keys[idx] = 0
                continue
            sub = counts[idx]
            # sorted mode tuples of depth k (repeat mode m counts[m] times)
            rows = np.repeat(np.arange(len(idx)), sub.sum(axis=1))
            modes = np.nonzero(sub)[1]
            reps = sub[sub > 0]
            tup = np.repeat(modes, reps).reshape(len(idx), k)
            keys[idx] = self._rank(tup, int(k)) + self.offsets[k]
            del rows
        return keys

    @staticmethod
    def _tuples(counts, depth):
        """Sorted mode tuples of all rows laid end to end: (row, mode, position
        in the row's tuple) of every entry and the start of each row."""
        N = counts.shape[0]
        row, mode = np.nonzero(counts)
        reps = counts[row, mode].astype(np.int64)
        row_t = np.repeat(row, reps)
        c = np.repeat(mode.astype(np.int64), reps)
        start = np.zeros(N + 1, dtype=np.int64)
        np.cumsum(depth, out=start[1:])
        i = np.arange(len(c), dtype=np.int64) - start[row_t]
        return row_t, c, i, start

    def _keys_int64(self, counts, depth):
        """keys_from_counts for every depth at once (int64 keys): each row's
        rank is a difference of running sums of its per-position binomial
        terms."""
        return self._keys_int64_from(*self._tuples(counts, depth), depth)

    def _keys_int64_from(self, row_t, c, i, start, depth):
        """The int64 keys of rows given as their sorted mode tuples laid end to
        end (the layout of _tuples)."""
        k = depth[row_t]
        n = self.M + k - 1
        b = c + i
        prev = np.empty_like(b)
        prev[1:] = b[:-1]
        prev[i == 0] = -1
        B = self.binom64
        term = B[n - 1 - prev, k - i] - B[n - b, k - i]
        cs = np.zeros(len(term) + 1, dtype=np.int64)
        np.cumsum(term, out=cs[1:])
        keys = cs[start[1:]] - cs[start[:-1]]
        off = np.asarray(self.offsets, dtype=np.int64)
        return keys + np.where(depth > 0, off[np.minimum(depth, len(off) - 1)], 0)

    def sort_keys(self, counts):
        """Keys whose order is the aux order and whose equality is aux equality,
        in a fixed-width numpy dtype: the global ranks when they fit in int64,
        else byte strings of the depth followed by the sorted mode tuple
        (big-endian, so that byte order is the reference's order: depth first,
        then lexicographic)."""
        counts = np.asarray(counts)
        if self.use_int64:
            return self.keys_from_counts(counts)
        depth = counts.sum(axis=1).astype(np.int64)
        if depth.size and depth.max() > self.D:
            raise AuxError("aux deeper than MAXHIER")
        row_t, c, i, _ = self._tuples(counts, depth)
        w = ">u2" if self.M < (1 << 16) else ">u4"
        arr = np.zeros((counts.shape[0], self.D + 1), dtype=w)
        arr[:, 0] = depth
        arr[row_t, 1 + i] = c
        return np.ascontiguousarray(arr).view(f"S{arr.itemsize * (self.D + 1)}").ravel()

    def keys_from_tuples(self, tup, depth):
        """sort_keys of aux given as sorted mode tuples: tup [N, W] with W at
        least the largest depth; the entries of row r beyond depth[r] are
        ignored.  Equal to sort_keys of the same aux as count rows."""
        depth = np.asarray(depth, dtype=np.int64)
        tup = np.asarray(tup, dtype=np.int64).reshape(len(depth), -1)
        if depth.size and depth.max() > self.D:
            raise AuxError("aux deeper than MAXHIER")
        mask = np.arange(tup.shape[1])[None, :] < depth[:, None]
        if self.use_int64:
            row_t, i = np.nonzero(mask)
            start = np.zeros(len(depth) + 1, dtype=np.int64)
            np.cumsum(depth, out=start[1:])
            return self._keys_int64_from(row_t, tup[row_t, i], i, start, depth)
        w = ">u2" if self.M < (1 << 16) else ">u4"
        arr = np.zeros((len(depth), self.D + 1), dtype=w)
        arr[:, 0] = depth
        k = min(tup.shape[1], self.D)
        arr[:, 1:1 + k] = np.where(mask[:, :k], tup[:, :k], 0)
        return np.ascontiguousarray(arr).view(f"S{arr.itemsize * (self.D + 1)}").ravel()

    def _rank(self, tup, k):
        n = self.M + k - 1
        b = tup.astype(np.int64) + np.arange(k, dtype=np.int64)[None, :]
        if self.use_int64:
            B = self.binom64
            r = np.zeros(len(tup), dtype=np.int64)
            prev = np.full(len(tup), -1, dtype=np.int64)
            for i in range(k):
                r += B[n - 1 - prev, k - i] - B[n - b[:, i], k - i]
                prev = b[:, i]
            return r
        B = self.binom
        r = np.zeros(len(tup), dtype=object)
        prev = np.full(len(tup), -1, dtype=np.int64)
        for i in range(k):
            r = r + B[n - 1 - prev, k - i] - B[n - b[:, i], k - i]
            prev = b[:, i]
        return r


def triangular_counts(n_mode, maxhier):
    """Count matrix of every aux with depth <= maxhier, in reference order."""
    blocks = [np.zeros((1, n_mode), dtype=np.int16)]
    # sorted tuples of depth k in lexicographic order, built from depth k-1 by
    # appending every mode >= the last one (hops_hierarchy.py:340-368)
    prev = np.zeros((1, 0), dtype=np.int32)
    for k in range(1, maxhier + 1):
        last = prev[:, -1] if k > 1 else np.zeros(1, dtype=np.int32)
        cnt = n_mode - last
        rep = np.repeat(np.arange(len(prev)), cnt)
        starts = np.repeat(last, cnt)
        offs = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
        new_last = (starts + offs).astype(np.int32)
        cur = np.concatenate([prev[rep], new_last[:, None]], axis=1)
        c = np.zeros((len(cur), n_mode), dtype=np.int16)
        np.add.at(c, (np.repeat(np.arange(len(cur)), k), cur.ravel()), 1)
        blocks.append(c)
        prev = cur
    return np.concatenate(blocks, axis=0)


def apply_static_filters(counts, filters, n_mode):
    """STATIC_FILTERS of basis/hierarchy_functions.py:7-140 on a count matrix."""
    keep = np.ones(len(counts), dtype=bool)
    total = counts.sum(axis=1)
    for item in filters:
        name, param = item[0], item[1]
        if name == "Triangular":
            mask = np.asarray(param[0], dtype=bool)
            if len(mask) != n_mode:
                raise UnsupportedRequest("The number of entries in the list of static filter "
                                         "booleans does not match the number of hierarchy "
                                         "modes", "hierarchy_static_filter", override=True)
            keep &= counts[:, mask].sum(axis=1) <= param[1]
        elif name == "LongEdge":
            mask = np.asarray(param[0], dtype=bool)
            if len(mask) != n_mode:
                raise UnsupportedRequest("The number of entries in the list of static filter "
                                         "booleans does not match the number of hierarchy "
                                         "modes", "hierarchy_static_filter", override=True)
            keep &= ((total <= param[1]) | (counts[:, mask].sum(axis=1) == 0)
                     | ((counts > 0).sum(axis=1) <= 1))
        elif name == "Markovian":
            mask = np.asarray(param, dtype=bool)
            if len(mask) != n_mode:
                raise UnsupportedRequest("The number of entries in the list of static filter "
                                         "booleans does not match the number of hierarchy "
                                         "modes", "hierarchy_static_filter", override=True)
            touches = (counts[:, mask] > 0).any(axis=1)
            keep &= (total == 0) | ~(touches & (total > 1))
        else:
            raise UnsupportedRequest(name, "hierarchy_static_filter")
    return counts[keep]


_PAD = np.iinfo(np.int64).max   # mode-tuple padding, above every mode index


def tuples_of(counts, width):
    """Sorted mode tuples of count rows, padded with _PAD to ``width``, and the
    rows' depths."""
    counts = np.asarray(counts)
    depth = counts.sum(axis=1).astype(np.int64)
    row_t, c, i, _ = AuxKeyer._tuples(counts, depth)
    tup = np.full((len(counts), max(int(width), 1)), _PAD, dtype=np.int64)
    tup[row_t, i] = c
    return tup, depth


def insert_mode(tup, m):
    """The sorted tuples tup [n, W] with mode m[i] inserted into row i (row i
    must have a free slot)."""
    m = np.asarray(m, dtype=np.int64)[:, None]
    pos = (tup <= m).sum(axis=1, keepdims=True)
    ar = np.arange(tup.shape[1])[None, :]
    right = np.full_like(tup, _PAD)
    right[:, 1:] = tup[:, :-1]
    return np.where(ar < pos, tup, np.where(ar == pos, m, right))


def remove_mode(tup, m):
    """The sorted tuples tup [n, W] with one occurrence of mode m[i] (which row
    i must hold) removed from row i."""
    m = np.asarray(m, dtype=np.int64)[:, None]
    pos = (tup < m).sum(axis=1, keepdims=True)
    ar = np.arange(tup.shape[1])[None, :]
    left = np.full_like(tup, _PAD)
    left[:, :-1] = tup[:, 1:]
    return np.where(ar < pos, tup, left)


class AuxBasis:
    """A sorted aux list with its up/down connection tables.

    counts: [n_hier, n_mode_abs] aux count matrix (absolute modes).
    modes:  sorted absolute modes of the current mode basis (relative index =
            position in this list); connections are built along these modes.
    """

    def __init__(self, counts, keyer, maxhier, modes=None):
        counts = np.asarray(counts)
        # sorted mode tuple of every aux (padded with _PAD beyond its depth),
        # from which its key is formed
        tup, depth = tuples_of(counts, maxhier)
        keys = keyer.keys_from_tuples(tup, depth)
        order = np.argsort(keys, kind="stable")
        self.counts = counts[order]
        self.keys = keys[order]
        self.tup = tup[order]
        if len(self.keys) == 0 or self.counts[0].sum() != 0:
            raise AuxError("Zero Vector not contained in list_aux!")
        self.keyer = keyer
        self.maxhier = maxhier
        self.n_hier = len(self.counts)
        n_mode_abs = self.counts.shape[1]
        self.modes = np.arange(n_mode_abs) if modes is None else np.asarray(modes, dtype=np.int64)
        self.depth = depth[order]
        self._build_connections()

    def index_of(self, counts):
        """Indices of the given aux (count rows) in this basis, -1 if absent."""
        return self.index_of_keys(self.keyer.sort_keys(counts))

    def index_of_keys(self, k):
        """Indices of the aux with the given sort keys in this basis, -1 if absent."""
        pos = np.searchsorted(self.keys, k)
        pos = np.minimum(pos, self.n_hier - 1)
        found = self.keys[pos] == k
        return np.where(found, pos, -1).astype(np.int64)

    def _build_connections(self):
        """k+1 / k-1 connections along the basis modes (hops_hierarchy.py:470-523).

        The candidate a + e_m of every aux below MAXHIER and basis mode m is
        its sorted mode tuple with m inserted in order; the candidates are
        keyed from those tuples (keys_from_tuples) and looked up in the
        basis's sorted keys, without forming their count rows."""
        ups_a, ups_u, ups_m = [], [], []
        below = np.nonzero(self.depth < self.maxhier)[0]
        nm = len(self.modes)
        if len(below) and nm:
            T = self.tup[below]
            D = T.shape[1]
            dep1 = self.depth[below] + 1
            Tsh = np.full_like(T, _PAD)          # the tuple shifted one place right
            Tsh[:, 1:] = T[:, :-1]
            ar = np.arange(D)
            # modes per batch: keep the candidate tuples near 4M entries
            per = max(1, int(4_000_000 // max(1, len(below) * D)))
            for c0 in range(0, nm, per):
                rels = np.arange(c0, min(c0 + per, nm))
                mabs = self.modes[rels].astype(np.int64)
                pos = (T[:, None, :] <= mabs[None, :, None]).sum(axis=2)
                cand = np.where(ar < pos[..., None], T[:, None, :],
                                np.where(ar == pos[..., None], mabs[None, :, None],
                                         Tsh[:, None, :]))
                keys = self.keyer.keys_from_tuples(cand.reshape(-1, D),
                                                   np.repeat(dep1, len(rels)))
                p = np.minimum(np.searchsorted(self.keys, keys), self.n_hier - 1)
                idx = np.where(self.keys[p] == keys, p, -1).reshape(len(below), len(rels))
                ii, jj = np.nonzero(idx >= 0)
                ups_a.append(below[ii])
                ups_u.append(idx[ii, jj])
                ups_m.append(rels[jj])
        if ups_a:
            a = np.concatenate(ups_a)
            u = np.concatenate(ups_u)
            m = np.concatenate(ups_m)
        else:
            a = u = m = np.zeros(0, dtype=np.int64)
        o = np.lexsort((m, a))
        self.up_a, self.up_u, self.up_m = a[o], u[o], m[o]
        o = np.lexsort((m, u))
        self.dn_a, self.dn_d, self.dn_m = u[o], a[o], m[o]
        # depth of the higher aux in the connecting mode (k_m(a) of the down term)
        self.dn_k = self.counts[self.dn_a, self.modes[self.dn_m]].astype(np.int64)
        self.up_ptr = np.zeros(self.n_hier + 1, dtype=np.int64)
        np.add.at(self.up_ptr, self.up_a + 1, 1)
        self.up_ptr = np.cumsum(self.up_ptr)
        self.dn_ptr = np.zeros(self.n_hier + 1, dtype=np.int64)
        np.add.at(self.dn_ptr, self.dn_a + 1, 1)
        self.dn_ptr = np.cumsum(self.dn_ptr)

    def first_level(self):
        """(aux index, relative mode) of every depth-1 aux along a basis mode."""
        if len(self.modes) == 0:
            return []
        e = np.zeros((len(self.modes), self.counts.shape[1]), dtype=self.counts.dtype)
        e[np.arange(len(self.modes)), self.modes] = 1
        idx = self.index_of(e)
        return [(int(i), rel) for rel, i in enumerate(idx) if i >= 0]


def triangular_basis(n_mode, maxhier, static_filters=()):
    keyer = AuxKeyer(n_mode, maxhier)
    counts = triangular_counts(n_mode, maxhier)
    if static_filters:
        counts = apply_static_filters(counts, static_filters, n_mode)
    return AuxBasis(counts, keyer, maxhier)


class TriangularHierarchy:
    """The full triangular hierarchy over ``n_mode`` modes to depth
    ``maxhier`` when its tables are built on the GPU
    (device.build_tables_triangular); the host count matrix is produced only
    when asked for (``counts``)."""

    def __init__(self, n_mode, maxhier):
        self.maxhier = int(maxhier)
        self.n_mode = int(n_mode)
        self.n_hier = comb(self.n_mode + self.maxhier, self.maxhier)
        self.modes = np.arange(self.n_mode)
        self._counts = None

    @property
    def counts(self):
        if self._counts is None:
            self._counts = triangular_counts(self.n_mode, self.maxhier)
        return self._counts
