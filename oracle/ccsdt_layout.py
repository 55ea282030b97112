"""ccq's compressed CCSDt T vector, restated in numpy (test infrastructure only).

Follows the reference's ``get_t_sizes_act`` (``src/utils/cc_utils.f90:560-630``:
the pos(6..16) offsets) and the sub-block declarations of the active-space
updates (``src/cc_opt_ccsdt/t2B0000_update_opt.f:48-57``, the same in every
``*_update_opt.f``): ten slices of the four T3 spin blocks, each in its block's
own axis order, concatenated after T1A, T1B, T2A, T2B, T2C.  Used by the tests
as the checker of ``ccq_b200_t_compress`` / ``ccq_b200_t_expand``.
"""
from __future__ import annotations

import itertools

import numpy as np


def ranges(froz, occ_a, occ_b, orbs, m1, m2):
    """Fortran bounds (lo, hi), 1-based inclusive, of the full blocks and the ten sub-blocks."""
    N0, N1, N2, N3 = froz, occ_a, occ_b, orbs
    va, vb, oa, ob = (N1 + 1, N3), (N2 + 1, N3), (N0 + 1, N1), (N0 + 1, N2)
    full = {'T3A': [va, va, va, oa, oa, oa], 'T3B': [vb, va, va, ob, oa, oa],
            'T3C': [vb, vb, va, ob, ob, oa], 'T3D': [vb, vb, vb, ob, ob, ob]}
    avA, avB, iv = (N1 + 1, m2), (N2 + 1, m2), (m2 + 1, N3)
    aoA, aoB, io = (m1 + 1, N1), (m1 + 1, N2), (N0 + 1, m1)
    subs = [('T3A', [va, va, avA, oa, oa, aoA]),
            ('T3B', [vb, va, avA, ob, oa, aoA]),
            ('T3B', [avB, iv, iv, aoB, io, io]),
            ('T3B', [avB, iv, iv, ob, oa, aoA]),
            ('T3B', [vb, va, avA, aoB, io, io]),
            ('T3C', [vb, avB, va, ob, aoB, oa]),
            ('T3C', [iv, iv, avA, io, io, aoA]),
            ('T3C', [iv, iv, avA, ob, aoB, oa]),
            ('T3C', [vb, avB, va, io, io, aoA]),
            ('T3D', [vb, vb, avB, ob, ob, aoB])]
    return full, subs


def pos_offsets(froz, occ_a, occ_b, orbs, m1, m2):
    """pos(1..16) of get_t_sizes_act, 1-based, as the reference computes them."""
    nocc_a, nocc_b = occ_a - froz, occ_b - froz
    nunocc_a, nunocc_b = orbs - occ_a, orbs - occ_b
    non_actocc, non_actunocc = m1 - froz, orbs - m2
    actocc_a, actocc_b = occ_a - m1, occ_b - m1
    actunocc_a, actunocc_b = m2 - occ_a, m2 - occ_b
    pos = [1]
    pos.append(pos[-1] + nocc_a * nunocc_a)
    pos.append(pos[-1] + nocc_b * nunocc_b)
    pos.append(pos[-1] + nocc_a * nocc_a * nunocc_a * nunocc_a)
    pos.append(pos[-1] + nocc_a * nocc_b * nunocc_a * nunocc_b)
    pos.append(pos[-1] + nocc_b * nocc_b * nunocc_b * nunocc_b)
    pos.append(pos[-1] + nunocc_a * nunocc_a * actunocc_a * nocc_a * nocc_a * actocc_a)
    pos.append(pos[-1] + nunocc_b * nunocc_a * actunocc_a * nocc_b * nocc_a * actocc_a)
    pos.append(pos[-1] + actunocc_b * non_actunocc * non_actunocc * actocc_b * non_actocc * non_actocc)
    pos.append(pos[-1] + actunocc_b * non_actunocc * non_actunocc * nocc_b * nocc_a * actocc_a)
    pos.append(pos[-1] + nunocc_b * nunocc_a * actunocc_a * actocc_b * non_actocc * non_actocc)
    pos.append(pos[-1] + nunocc_b * actunocc_b * nunocc_a * nocc_b * actocc_b * nocc_a)
    pos.append(pos[-1] + non_actunocc * non_actunocc * actunocc_a * non_actocc * non_actocc * actocc_a)
    pos.append(pos[-1] + non_actunocc * non_actunocc * actunocc_a * nocc_b * actocc_b * nocc_a)
    pos.append(pos[-1] + nunocc_b * actunocc_b * nunocc_a * non_actocc * non_actocc * actocc_a)
    pos.append(pos[-1] + nunocc_b * nunocc_b * actunocc_b * nocc_b * nocc_b * actocc_b)
    return pos


def _n(r):
    return max(r[1] - r[0] + 1, 0)


def full_blocks(t_full, dims, t12):
    """The four T3 blocks of a full T vector as Fortran-ordered arrays (views)."""
    froz, occ_a, occ_b, orbs = dims
    full, _ = ranges(froz, occ_a, occ_b, orbs, froz, occ_a)
    out, off = {}, t12
    for b in ('T3A', 'T3B', 'T3C', 'T3D'):
        shp = [_n(r) for r in full[b]]
        n = int(np.prod(shp))
        out[b] = t_full[off:off + n].reshape(shp, order='F')
        off += n
    return out


def t12_size(froz, occ_a, occ_b, orbs):
    return pos_offsets(froz, occ_a, occ_b, orbs, froz, occ_a)[5] - 1


def compress(t_full, dims, m1, m2):
    froz, occ_a, occ_b, orbs = dims
    full, subs = ranges(froz, occ_a, occ_b, orbs, m1, m2)
    t12 = t12_size(*dims)
    blocks = full_blocks(t_full, dims, t12)
    parts = [t_full[:t12]]
    for b, rr in subs:
        sl = tuple(slice(r[0] - f[0], r[1] - f[0] + 1) if _n(r) else slice(0, 0) for r, f in zip(rr, full[b]))
        parts.append(blocks[b][sl].ravel(order='F'))
    return np.concatenate(parts)


GROUPS = {'T3A': [(0, 1, 2), (3, 4, 5)], 'T3B': [(1, 2), (4, 5)], 'T3C': [(0, 1), (3, 4)], 'T3D': [(0, 1, 2), (3, 4, 5)]}


def _sign(p):
    s = 1
    for x in range(len(p)):
        for y in range(x + 1, len(p)):
            if p[y] < p[x]:
                s = -s
    return s


def expand(t_act, dims, m1, m2):
    froz, occ_a, occ_b, orbs = dims
    full, subs = ranges(froz, occ_a, occ_b, orbs, m1, m2)
    t12 = t12_size(*dims)
    n_full = t12 + sum(int(np.prod([_n(r) for r in full[b]])) for b in full)
    out = np.zeros(n_full)
    out[:t12] = t_act[:t12]
    blocks = full_blocks(out, dims, t12)
    off = t12
    for b, rr in subs:
        shp = [_n(r) for r in rr]
        n = int(np.prod(shp))
        sub = t_act[off:off + n].reshape(shp, order='F')
        off += n
        if not n:
            continue
        g0, g1 = GROUPS[b]
        for p0 in itertools.permutations(range(len(g0))):
            for p1 in itertools.permutations(range(len(g1))):
                axes = list(range(6))
                for k in range(len(g0)):
                    axes[g0[k]] = g0[p0[k]]
                for k in range(len(g1)):
                    axes[g1[k]] = g1[p1[k]]
                # the element at x goes to y with y[g[k]] = x[g[p[k]]]: index arrays per output axis
                idx = np.indices(shp)
                tgt = [idx[axes[k]] + (rr[axes[k]][0] - full[b][k][0]) for k in range(6)]
                blocks[b][tuple(tgt)] = _sign(p0) * _sign(p1) * sub
    return out
