"""Determinant-space coupled-cluster residuals (test infrastructure only).

This is the equation-free check of the oracle: the CC residual
``R_mu = <Phi_mu| exp(-T) H exp(T) |Phi>`` and the correlation energy are
evaluated by applying second-quantised operators to Fock-space vectors
(Jordan-Wigner signs on bit strings).  No derived CC equations enter, so it
pins the symbolic residuals of ``ccq_b200.eqgen.wick`` independently of the
reference's generated diagram code (``src/cc/t*_update.f90``), whose residual
is the same projection.  Only tiny systems (<= ~12 spin orbitals) are feasible.

Spin-orbital order: occupied first, then virtual; ``t_n`` is stored as
``t[a0..a_{n-1}, i0..i_{n-1}]`` with virtual indices counted from 0.
Only ``tests/`` use this module.
"""
from __future__ import annotations

import itertools
import numpy as np


class FockSpace:
    def __init__(self, nso):
        self.n = nso
        self.states = np.arange(1 << nso, dtype=np.int64)

    def _parity_below(self, p):
        mask = (1 << p) - 1
        x = self.states & mask
        # popcount parity
        c = np.zeros_like(x)
        y = x.copy()
        while np.any(y):
            c ^= (y & 1)
            y >>= 1
        return 1 - 2 * c

    def prepare(self):
        self.sgn = [self._parity_below(p) for p in range(self.n)]
        self.occ = [((self.states >> p) & 1).astype(bool) for p in range(self.n)]

    def ann(self, p, vec):
        out = np.zeros_like(vec)
        m = self.occ[p]
        src = self.states[m]
        out[src ^ (1 << p)] += self.sgn[p][m] * vec[m]
        return out

    def cre(self, p, vec):
        out = np.zeros_like(vec)
        m = ~self.occ[p]
        src = self.states[m]
        out[src ^ (1 << p)] += self.sgn[p][m] * vec[m]
        return out

    def string(self, ops, vec):
        """Apply ops (list of (p, is_creator)) right-to-left like operator algebra."""
        for p, c in reversed(ops):
            vec = self.cre(p, vec) if c else self.ann(p, vec)
            if not np.any(vec):
                return vec
        return vec


class DetCC:
    """Exact projective CC machinery on a Fock space of ``nso`` spin orbitals."""

    def __init__(self, h, v, nocc):
        # h: (N,N) core one-body; v: (N,N,N,N) antisymmetrised <pq||rs>
        self.h = h
        self.v = v
        self.N = h.shape[0]
        self.O = nocc
        self.V = self.N - nocc
        self.fs = FockSpace(self.N)
        self.fs.prepare()
        self.phi = np.zeros(1 << self.N)
        self.phi[(1 << nocc) - 1] = 1.0

    def apply_h(self, vec):
        fs = self.fs
        N = self.N
        out = np.zeros_like(vec)
        for p in range(N):
            for q in range(N):
                c = self.h[p, q]
                if c != 0.0:
                    out += c * fs.string([(p, True), (q, False)], vec)
        # 1/4 v_pqrs p+ q+ s r  = sum_{p<q, r<s} v_pqrs p+ q+ s r
        for p in range(N):
            for q in range(p + 1, N):
                tmp = None
                for r in range(N):
                    for s in range(r + 1, N):
                        c = self.v[p, q, r, s]
                        if c == 0.0:
                            continue
                        w = fs.string([(s, False), (r, False)], vec)
                        tmp = c * w if tmp is None else tmp + c * w
                if tmp is not None:
                    out += fs.string([(p, True), (q, True)], tmp)
        return out

    def apply_t(self, ts, vec, sign=1.0):
        """T = sum_n sum_{unique} t_n a0+..a_{n-1}+ i_{n-1}..i0 applied to vec."""
        fs = self.fs
        O = self.O
        out = np.zeros_like(vec)
        for n, t in ts.items():
            for occ in itertools.combinations(range(O), n):
                base = fs.string([(i, False) for i in reversed(occ)], vec)
                if not np.any(base):
                    continue
                for vir in itertools.combinations(range(self.V), n):
                    c = t[vir + occ]
                    if c == 0.0:
                        continue
                    out += sign * c * fs.string([(O + a, True) for a in vir], base)
        return out

    def exp_t(self, ts, vec, sign=1.0):
        res = vec.copy()
        term = vec.copy()
        for k in range(1, 2 * self.N + 2):
            term = self.apply_t(ts, term, sign) / k
            if not np.any(np.abs(term) > 0):
                break
            res += term
        return res

    def sim_vector(self, ts):
        w = self.exp_t(ts, self.phi, 1.0)
        w = self.apply_h(w)
        return self.exp_t(ts, w, -1.0)

    def e_ref(self):
        return float(self.phi @ self.apply_h(self.phi))

    def residual(self, ts, level, w=None):
        """Dense antisymmetric residual R[a0.., i0..] of excitation ``level``."""
        if w is None:
            w = self.sim_vector(ts)
        O, V = self.O, self.V
        R = np.zeros((V,) * level + (O,) * level)
        fs = self.fs
        for occ in itertools.combinations(range(O), level):
            base = fs.string([(i, False) for i in reversed(occ)], self.phi)
            for vir in itertools.combinations(range(V), level):
                ket = fs.string([(O + a, True) for a in vir], base)
                val = float(ket @ w)
                for po in itertools.permutations(range(level)):
                    so = _perm_sign(po)
                    for pv in itertools.permutations(range(level)):
                        sv = _perm_sign(pv)
                        R[tuple(vir[k] for k in pv) + tuple(occ[k] for k in po)] = so * sv * val
        return R

    def energy(self, ts):
        w = self.sim_vector(ts)
        return float(self.phi @ w) - self.e_ref()

    def fci_energy(self, nalpha_mask=None):
        """Lowest eigenvalue of H in the N-electron, Sz-of-reference sector minus E_ref."""
        fs = self.fs
        states = fs.states
        pc = np.array([bin(int(s)).count('1') for s in states])
        sel = np.where(pc == self.O)[0]
        if nalpha_mask is not None:
            a_mask, n_alpha = nalpha_mask
            na = np.array([bin(int(s) & a_mask).count('1') for s in states[sel]])
            sel = sel[na == n_alpha]
        H = np.zeros((len(sel), len(sel)))
        for k, s in enumerate(sel):
            e = np.zeros(1 << self.N)
            e[s] = 1.0
            H[:, k] = self.apply_h(e)[sel]
        w = np.linalg.eigvalsh(0.5 * (H + H.T))
        return float(w[0]) - self.e_ref()


def _perm_sign(p):
    p = list(p)
    s = 1
    for i in range(len(p)):
        for j in range(i + 1, len(p)):
            if p[j] < p[i]:
                s = -s
    return s
