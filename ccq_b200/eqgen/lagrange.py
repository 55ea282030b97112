"""Left (Lambda) CCSD and CR-CC(2,3) equations by differentiating the CC Lagrangian.

The reference solves the left CCSD equations with generated diagram routines
(``src/lcc/L1A_update.f`` .. ``L2C_update.f``, driven by ``update_l2`` in
``src/update_lcc.f90:10-104``) and builds the triples moments and left
projections for CR-CC(2,3) with ``src/mm_cor/mm_t3a..d.f`` and
``src/lcc/L3A..L3D_update.f`` (``crcc23``, ``src/mm_correct.f90:11-344``).
The same quantities follow from the Lagrangian

    L(T, Lambda) = E(T) + sum_n sum_{unique mu in n} lambda_mu R_mu(T)

with ``R_mu = <mu| exp(-T) H exp(T) |Phi>`` (the residuals of ``wick``):

  * left residual   LH_mu = dL / dt_mu          (mu singles, doubles; T = T1 + T2)
                          = <Phi|(1 + Lambda)(Hbar - E)|mu>, which vanishes at
                          the left solution (the reference's ``update_l2``
                          residual: disconnected lambda1 * Hbar1 products
                          included, the lambda_mu E_cor term excluded);
  * triples moment  M_mu  = R_mu(T1, T2, T3 = 0)  (mu triples);
  * left projection l_mu  = dL / dt3_mu at T3 = 0 = <Phi|(1 + Lambda) Hbar|mu>.

Differentiating a term with respect to the unique amplitude t_mu removes one
factor t_m and sums the result over the (m!)^2 signed permutations of the
removed factor's labels (every stored copy of t_mu).  Terms are returned in
``wick``'s format, ``(Fraction coef, [vertex, factors...])``, with external
labels ``a0.., i0..`` and amplitude factors named ``t<n>`` / ``l<n>``.
"""
from __future__ import annotations

from fractions import Fraction
from functools import lru_cache
from itertools import permutations
from math import factorial

from . import wick


def _perm_sign(p):
    return wick._parity(list(p))


def _rename_all(tensors, taken):
    """Rename every label of ``tensors`` to fresh dummies (o*/v*) not in ``taken``."""
    m = {}
    cnt = {'o': 0, 'v': 0}
    for _, ls in tensors:
        for l in ls:
            if l in m:
                continue
            sp = 'o' if l[0] in 'io' else 'v'
            while f'{sp}{cnt[sp]}' in taken:
                cnt[sp] += 1
            m[l] = f'{sp}{cnt[sp]}'
            cnt[sp] += 1
    return [(nm, tuple(m[l] for l in ls)) for nm, ls in tensors]


def _derivative(coef, tensors, m):
    """Terms of d(coef * prod tensors)/dt_m for one unique amplitude of rank m.

    Each occurrence of ``t<m>`` is removed in turn; its labels become the
    external labels (virtual a0.., occupied i0..) and the result is summed
    over the signed permutations of those labels.  Other labels are dummies.
    """
    name = f't{m}'
    out = []
    for k, (nm, ls) in enumerate(tensors):
        if nm != name:
            continue
        vl, ol = ls[:m], ls[m:]
        ext = {l: f'a{q}' for q, l in enumerate(vl)}
        ext.update({l: f'i{q}' for q, l in enumerate(ol)})
        rest = [t for q, t in enumerate(tensors) if q != k]
        # dummies first to fresh names that cannot collide with a*/i*
        dm = {}
        cnt = {'o': 0, 'v': 0}
        for _, lls in rest:
            for l in lls:
                if l in ext or l in dm:
                    continue
                sp = 'o' if l[0] in 'io' else 'v'
                dm[l] = f'{sp}{cnt[sp]}'
                cnt[sp] += 1
        base = [(nm2, tuple(ext.get(l, dm.get(l)) for l in lls)) for nm2, lls in rest]
        occ = [f'i{q}' for q in range(m)]
        vir = [f'a{q}' for q in range(m)]
        for pv in permutations(range(m)):
            for po in permutations(range(m)):
                s = _perm_sign(pv) * _perm_sign(po)
                mp = {vir[q]: vir[pv[q]] for q in range(m)}
                mp.update({occ[q]: occ[po[q]] for q in range(m)})
                out.append((coef * s, [(nm2, tuple(mp.get(l, l) for l in lls)) for nm2, lls in base]))
    return out


def _merge(terms):
    acc = {}
    for c, tensors in terms:
        key, s = wick.canonical(tensors)
        if key is None:
            continue
        acc[key] = acc.get(key, Fraction(0)) + c * s
    out = [(c, [key[0]] + list(key[1])) for key, c in acc.items() if c != 0]
    out.sort(key=lambda t: wick._key_rank((t[1][0], tuple(t[1][1:]))))
    return out


def _lagrangian_products(tranks, levels, lam_levels):
    """Unmerged Lagrangian terms: energy + sum_n (1/n!^2) lambda_n[a.., i..] R_n[a.., i..].

    The residual's external labels are renamed to dummies, so every label of a
    Lagrangian term is summed.
    """
    out = []
    for c, tensors in wick.energy_terms():
        out.append((c, list(tensors)))
    for n in lam_levels:
        lam = (f'l{n}', tuple(f'a{q}' for q in range(n)) + tuple(f'i{q}' for q in range(n)))
        w = Fraction(1, factorial(n) ** 2)
        for c, tensors in wick.residual_terms(n, tranks):
            prod = list(tensors) + [lam]
            out.append((c * w, _rename_all(prod, set())))
    return out


@lru_cache(maxsize=None)
def left_residual_terms(level):
    """LH of excitation ``level`` (1 or 2) for Lambda-CCSD with bare f, v and explicit T1.

    Every term carries a bare Hamiltonian vertex (``f``/``v``, undressed) and
    any of ``t1``, ``t2``, ``l1``, ``l2``.
    """
    terms = []
    for c, tensors in _lagrangian_products((1, 2), (1, 2), (1, 2)):
        terms += _derivative(c, tensors, level)
    return _merge(terms)


@lru_cache(maxsize=None)
def triples_moment_terms():
    """M3 = <mu_3| (H1 exp(T2))_C |Phi> with T1-dressed f, v (CCSDT R3 at T3 = 0)."""
    return list(wick.residual_terms(3, (2,)))


@lru_cache(maxsize=None)
def triples_left_terms():
    """l3 = <Phi|(Lambda1 + Lambda2) Hbar|mu_3> with T1-dressed f, v, T2, lambda1, lambda2.

    The derivative of sum_n lambda_n R_n(T1, T2, T3) with respect to t3 at
    T3 = 0; R_n carries T1 through the dressed vertex.
    """
    terms = []
    for n in (1, 2):
        lam = (f'l{n}', tuple(f'a{q}' for q in range(n)) + tuple(f'i{q}' for q in range(n)))
        w = Fraction(1, factorial(n) ** 2)
        for c, tensors in wick.residual_terms(n, (2, 3)):
            if sum(1 for nm, _ in tensors if nm == 't3') != 1:
                continue
            prod = _rename_all(list(tensors) + [lam], set())
            terms += _derivative(c * w, prod, 3)
    return _merge(terms)
