"""Spin-orbital coupled-cluster residual equations by Wick's theorem.

The reference machine-generates its diagram routines (``src/cc/t*_update.f90``) as
long Fortran loop nests.  This module derives the same residuals symbolically, as
data, so that one plan compiler can lower them to GPU contraction kernels.

Formulation.  The Hamiltonian is similarity-transformed by T1 first
(``H1 = exp(-T1) H exp(T1)``), which keeps it a two-body operator with dressed
one-body ``f`` and antisymmetrised two-body ``v`` elements.  The residual of
excitation level ``m`` is then

    R^{a0..}_{i0..} = < Phi_{i0..}^{a0..} | (H1 exp(T2 + T3 + T4))_C | Phi >

which equals ``<mu| exp(-T) H exp(T) |Phi>`` because all cluster operators
commute.  The Jacobi step of the reference (``src/cc/t1A_update.f90:518-525``,
``src/cc/t2A_update.f90:1885-1901``) consumes exactly this residual.

Conventions (fixed here, validated numerically against the determinant-space
oracle):
  * ``|Phi_{i0..}^{a0..}> = a0^+ .. a_{m-1}^+ i_{m-1} .. i0 |Phi>``
  * ``T_n = (1/n!)^2 sum t[a0..a_{n-1}, i0..i_{n-1}] a0^+..a_{n-1}^+ i_{n-1}..i0``
  * ``H1 = sum f[p,q] {p^+ q} + 1/4 sum v[p,q,r,s] {p^+ q^+ s r}``,
    ``v[p,q,r,s] = <pq||rs>``.

A term is ``coef * f|v[...] * prod t_n[...]`` with external labels ``i0..``,
``a0..`` and dummy labels ``o0..`` (occupied) and ``v0..`` (virtual).
"""
from __future__ import annotations

from fractions import Fraction
from itertools import permutations, product, combinations_with_replacement
from math import factorial
from functools import lru_cache

# ---------------------------------------------------------------------------
# operator strings
# ---------------------------------------------------------------------------
# An operator is (string_id, space, is_creator, label).  Quasi-annihilators are
# virtual annihilators and occupied creators; quasi-creators are the others.


def _is_qann(op):
    _, space, cre, _ = op
    return (space == 'v' and not cre) or (space == 'o' and cre)


def _parity(seq):
    inv = 0
    n = len(seq)
    for i in range(n):
        si = seq[i]
        for j in range(i + 1, n):
            if seq[j] < si:
                inv += 1
    return -1 if inv & 1 else 1


def _h_parts(kind):
    """All o/v space assignments of the one- or two-body vertex."""
    if kind == 'f':
        return [('f', sp) for sp in product('ov', repeat=2)]
    return [('v', sp) for sp in product('ov', repeat=4)]


def _count_lines(hkind, spaces):
    """(quasi-creators, quasi-annihilators) of a vertex part."""
    if hkind == 'f':
        p, q = spaces
        ops = [(p, True), (q, False)]
    else:
        p, q, r, s = spaces
        ops = [(p, True), (q, True), (s, False), (r, False)]
    qann = sum(1 for sp, cre in ops if (sp == 'v' and not cre) or (sp == 'o' and cre))
    return len(ops) - qann, qann


def _enumerate(level, hkind, hspaces, tranks):
    """Yield (sign, hlabels, tlabels_list, ext_pairs) for canonical full contractions.

    T slots are filled in a fixed order, which picks one representative of
    every class of contractions related by relabelling a T's own lines; that
    multiplicity ((n!)^2 per T_n) cancels the (1/n!)^2 of the operator.
    """
    ops = []
    # bra <Phi| i0^+ .. i_{m-1}^+ a_{m-1} .. a0
    for k in range(level):
        ops.append(('B', 'o', True, f'i{k}'))
    for k in reversed(range(level)):
        ops.append(('B', 'v', False, f'a{k}'))
    if hkind == 'f':
        p, q = hspaces
        ops += [('H', p, True, 'hp'), ('H', q, False, 'hq')]
    else:
        p, q, r, s = hspaces
        ops += [('H', p, True, 'hp'), ('H', q, True, 'hq'), ('H', s, False, 'hs'), ('H', r, False, 'hr')]
    tslots = []  # per T: {'v': [positions in order], 'o': [...]}
    for ti, n in enumerate(tranks):
        sid = f'T{ti}'
        vpos, opos = [], []
        for k in range(n):
            vpos.append(len(ops))
            ops.append((sid, 'v', True, f't{ti}v{k}'))
        base = len(ops)
        for k in reversed(range(n)):
            ops.append((sid, 'o', False, f't{ti}o{k}'))
        # occupied slot k sits at base + (n-1-k)
        opos = [base + (n - 1 - k) for k in range(n)]
        tslots.append({'v': vpos, 'o': opos})
    nops = len(ops)
    qann = [i for i in range(nops) if _is_qann(ops[i])]
    qcre = [i for i in range(nops) if not _is_qann(ops[i])]
    if len(qann) != len(qcre):
        return
    used = [False] * nops
    tnext = [{'v': 0, 'o': 0} for _ in tranks]
    pairs = []

    def rec(idx):
        if idx == len(qann):
            yield list(pairs)
            return
        x = qann[idx]
        sx = ops[x][0]
        space = ops[x][1]
        # candidate partners: H quasi-creators (only for bra ops) and next free T slot
        if sx == 'B':
            for y in range(x + 1, nops):
                if ops[y][0] == 'H' and not used[y] and not _is_qann(ops[y]) and ops[y][1] == space:
                    used[y] = True
                    pairs.append((x, y))
                    yield from rec(idx + 1)
                    pairs.pop()
                    used[y] = False
        for ti in range(len(tranks)):
            sl = tslots[ti][space]
            k = tnext[ti][space]
            if k >= len(sl):
                continue
            y = sl[k]
            if y <= x:
                continue
            tnext[ti][space] += 1
            used[y] = True
            pairs.append((x, y))
            yield from rec(idx + 1)
            pairs.pop()
            used[y] = False
            tnext[ti][space] -= 1

    for prs in rec(0):
        # all quasi-creators used?
        usedset = set(y for _, y in prs)
        if len(usedset) != len(qcre):
            continue
        # connectivity: every T touches H
        touched = set()
        for x, y in prs:
            if ops[x][0] == 'H' and ops[y][0].startswith('T'):
                touched.add(ops[y][0])
        if len(touched) != len(tranks):
            continue
        seq = []
        for x, y in prs:
            seq += [x, y]
        sign = _parity(seq)
        # label identification
        lab = {}
        nd = {'o': 0, 'v': 0}
        for x, y in prs:
            lx = ops[x][3]
            ly = ops[y][3]
            if ops[x][0] == 'B':
                lab[ly] = lx
            else:
                sp = ops[x][1]
                d = f'{sp}{nd[sp]}'
                nd[sp] += 1
                lab[lx] = d
                lab[ly] = d
        for op in ops:
            if op[0] == 'B':
                lab[op[3]] = op[3]
        if hkind == 'f':
            hl = (lab['hp'], lab['hq'])
        else:
            hl = (lab['hp'], lab['hq'], lab['hr'], lab['hs'])
        tl = []
        for ti, n in enumerate(tranks):
            tl.append(tuple(lab[f't{ti}v{k}'] for k in range(n)) + tuple(lab[f't{ti}o{k}'] for k in range(n)))
        yield sign, hl, tl


# ---------------------------------------------------------------------------
# canonical forms
# ---------------------------------------------------------------------------

def _label_rank(l):
    kind = l[0]
    order = {'i': 0, 'a': 1, 'o': 2, 'v': 3}[kind]
    return (order, int(l[1:]))


def groups_of(name, rank):
    """Antisymmetric index groups of a tensor (positions)."""
    if name == 'f':
        return [(0,), (1,)]
    if name == 'v':
        return [(0, 1), (2, 3)]
    # amplitude t<n> / l<n>: (virtual..., occupied...)
    n = rank // 2
    return [tuple(range(n)), tuple(range(n, 2 * n))]


def _sort_groups(name, labels):
    labels = list(labels)
    sign = 1
    for g in groups_of(name, len(labels)):
        sub = [labels[p] for p in g]
        if len(set(sub)) != len(sub):
            return None, 0
        order = sorted(range(len(sub)), key=lambda q: _label_rank(sub[q]))
        sign *= _parity(order)
        for p, q in zip(g, order):
            labels[p] = sub[q]
    return tuple(labels), sign


def _relabel(tensors, m):
    return [(nm, tuple(m.get(l, l) for l in ls)) for nm, ls in tensors]


def canonical(tensors):
    """Canonical key and sign of a product under dummy relabelling and antisymmetry.

    ``tensors[0]`` is the Hamiltonian vertex; the remaining factors commute.
    Returns (key, sign) or (None, 0) if the product vanishes identically.
    """
    dummies = sorted({l for _, ls in tensors for l in ls if l[0] in 'ov'}, key=_label_rank)
    do = [l for l in dummies if l[0] == 'o']
    dv = [l for l in dummies if l[0] == 'v']
    best = None
    for po in permutations(range(len(do))):
        for pv in permutations(range(len(dv))):
            m = {do[i]: f'o{po[i]}' for i in range(len(do))}
            m.update({dv[i]: f'v{pv[i]}' for i in range(len(dv))})
            rel = _relabel(tensors, m)
            sign = 1
            out = []
            for nm, ls in rel:
                sl, s = _sort_groups(nm, ls)
                if sl is None:
                    return None, 0
                sign *= s
                out.append((nm, sl))
            key = (out[0], tuple(sorted(out[1:], key=lambda t: (t[0], [_label_rank(x) for x in t[1]]))))
            rk = _key_rank(key)
            if best is None or rk < best[0]:
                best = (rk, key, sign)
    return best[1], best[2]


def _key_rank(key):
    h, ts = key
    return ((h[0], [_label_rank(x) for x in h[1]]), [(t[0], [_label_rank(x) for x in t[1]]) for t in ts])


# ---------------------------------------------------------------------------
# residual generation
# ---------------------------------------------------------------------------

def _tprods(allowed, maxn=4):
    out = [()]
    for k in range(1, maxn + 1):
        out += list(combinations_with_replacement(allowed, k))
    return out


@lru_cache(maxsize=None)
def residual_terms(level, tranks_allowed):
    """Merged spin-orbital terms of the level-``level`` residual.

    ``tranks_allowed`` is the tuple of cluster ranks present besides T1 (e.g.
    ``(2,)`` for CCSD, ``(2, 3)`` for CCSDT).  Returns a list of
    ``(Fraction coef, tensors)`` with ``tensors[0]`` the ``f``/``v`` vertex.
    """
    acc = {}
    for hkind in ('f', 'v'):
        for _, hsp in _h_parts(hkind):
            ncre, nqann = _count_lines(hkind, hsp)
            for tp in _tprods(tranks_allowed):
                if len(tp) > nqann:
                    continue
                # open lines: H quasi-creators + T lines - contracted H quasi-annihilators
                if ncre + sum(2 * n for n in tp) - nqann != 2 * level:
                    continue
                if sum(2 * n for n in tp) < nqann:
                    continue
                # 1/k! for identical factors in the exponential
                mult = 1
                for r in set(tp):
                    mult *= factorial(tp.count(r))
                base = Fraction(1, 4) if hkind == 'v' else Fraction(1)
                base /= mult
                for sign, hl, tl in _enumerate(level, hkind, hsp, tp):
                    tensors = [(hkind, hl)] + [(f't{n}', l) for n, l in zip(tp, tl)]
                    key, s = canonical(tensors)
                    if key is None:
                        continue
                    acc[key] = acc.get(key, Fraction(0)) + base * sign * s
    out = []
    for key, c in acc.items():
        if c != 0:
            out.append((c, [key[0]] + list(key[1])))
    out.sort(key=lambda t: _key_rank((t[1][0], tuple(t[1][1:]))))
    return out


def ext_labels(level):
    return tuple(f'a{k}' for k in range(level)) + tuple(f'i{k}' for k in range(level))


def _orbit_key(args):
    level, tensors = args
    occ = [f'i{k}' for k in range(level)]
    vir = [f'a{k}' for k in range(level)]
    best = None
    for po in permutations(occ):
        for pv in permutations(vir):
            m = dict(zip(occ, po))
            m.update(zip(vir, pv))
            key, s = canonical(_relabel(tensors, m))
            rk = _key_rank(key)
            if best is None or rk < best[0]:
                best = (rk, key, s, m)
    return best[1], best[2], best[3]


def orbit_groups(level, terms, workers=None):
    """Group terms related by permutations of external labels.

    Returns a list of ``(base_tensors, [(perm_map, coef), ...])``: the term
    equals ``coef * base`` with every external label ``x`` of the base renamed
    to ``perm_map[x]``.  Evaluating ``base`` once per distinct spin pattern and
    adding the permuted copies is the antisymmetriser of the reference's
    generated code (its ``sum_stripe`` calls with permutation strings).
    ``workers`` > 1 spreads the search over processes (level 4 has 576
    external permutations per term).
    """
    args = [(level, tensors) for _, tensors in terms]
    if workers and workers > 1 and len(terms) > 50:
        import multiprocessing as mp
        with mp.get_context('spawn').Pool(workers) as pool:
            keys = pool.map(_orbit_key, args, chunksize=8)
    else:
        keys = [_orbit_key(a) for a in args]
    groups = {}
    order = []
    for (coef, tensors), (key, s, m) in zip(terms, keys):
        # tensors relabelled by m equals s * B  =>  tensors = s * (B relabelled by m^-1)
        inv = {v: k for k, v in m.items()}
        if key not in groups:
            groups[key] = []
            order.append(key)
        groups[key].append((inv, coef * s))
    return [([key[0]] + list(key[1]), groups[key]) for key in order]


def energy_terms():
    """Correlation energy <Phi|(H exp(T))_C|Phi> with undressed f, v and T1, T2.

    Mirrors ``calculate_unsorted_energy`` (``src/energy.f90:138-270``):
    E = sum f_ia t_ia + 1/4 sum v_ijab t_ijab + 1/2 sum v_ijab t_ia t_jb.
    """
    return [
        (Fraction(1), [('f', ('o0', 'v0')), ('t1', ('v0', 'o0'))]),
        (Fraction(1, 4), [('v', ('o0', 'o1', 'v0', 'v1')), ('t2', ('v0', 'v1', 'o0', 'o1'))]),
        (Fraction(1, 2), [('v', ('o0', 'o1', 'v0', 'v1')), ('t1', ('v0', 'o0')), ('t1', ('v1', 'o1'))]),
    ]


METHOD_TRANKS = {
    'CCSD': (2,),
    'CCSDT': (2, 3),
    'CCSDTQ': (2, 3, 4),
}


def method_levels(method):
    tr = METHOD_TRANKS[method]
    return (1,) + tr
