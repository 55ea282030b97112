"""CR-CC(2,3) oracles (test infrastructure only).

Two independent CPU restatements of the reference's CR-CC(2,3) chain
(``calc_type=CR-CC(2,3)``: ``hbar2`` ``src/hbar.f90:10-720``, ``solve_lcc``
``src/solve_cc.f90:101-173`` with ``update_l2``/``left_jacobi_update``
``src/update_lcc.f90:10-280`` and ``calculate_left_energy``
``src/energy.f90:103-136``, then ``crcc23``/``cal_d3``
``src/mm_correct.f90:11-481``):

``ExactCRCC`` works in determinant space (``oracle.detcc``): Hbar =
exp(-T) H exp(T) is applied to Fock-space vectors, the left CCSD equations
<Phi|(1 + Lambda)(Hbar - E)|mu> = 0 are solved by dense linear algebra,
M_mu = <mu|Hbar|Phi>, l_mu = <Phi|(1 + Lambda) Hbar|mu>, and the diagonal
pieces of Hbar (one-, two- and three-body) are read off expectation values
of 1- and 2-quasiparticle states.  No derived equations enter, so it pins
the physics; it is feasible for <= ~12 spin orbitals.

``DenseCRCC`` restates the reference's algorithm on dense spin-orbital
tensors: Hbar one- and two-body diagonals from T1-dressed integrals and T2,
the left iterations with the reference's Jacobi denominators
(``h1(a,a) - h1(i,i) - E_cor + shift``), its energy proxy
sqrt(sum LH^2) + E_cor and the shared DIIS driver (``oracle.solver``), the
moments and left projections from ``ccq_b200.eqgen.lagrange``, and the four
denominators of ``crcc23``: A (Fock), B (Hbar one-body), C (+ two-body) and
D (+ three-body ``cal_d3`` terms, including the reference's loop bound
``e = occ_a + 2 .. orbs`` in the beta-beta-beta term ``d3d1``,
``src/mm_correct.f90:455-463``, which skips the first occ_a - occ_b + 1 beta
virtuals).

Only ``tests/`` use this module.
"""
from __future__ import annotations

import itertools

import numpy as np

from ccq_b200.eqgen import lagrange, wick
from oracle import solver as S
from oracle.detcc import DetCC, _perm_sign

LETTERS = 'abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ'


def eval_terms(terms, level, amps, fmat, vmat, O):
    """Dense residual-like tensor [vir.., occ..] of a term list (einsum per term)."""
    N = fmat.shape[0]
    V = N - O
    sl = {'o': slice(0, O), 'v': slice(O, N)}
    sp = lambda l: 'o' if l[0] in 'io' else 'v'
    out = np.zeros((V,) * level + (O,) * level)
    ext = wick.ext_labels(level)
    for coef, tensors in terms:
        lab = {}
        ops, subs = [], []
        for name, ls in tensors:
            for l in ls:
                if l not in lab:
                    lab[l] = LETTERS[len(lab)]
            if name == 'f':
                arr = fmat[sl[sp(ls[0])], sl[sp(ls[1])]]
            elif name == 'v':
                arr = vmat[sl[sp(ls[0])], sl[sp(ls[1])], sl[sp(ls[2])], sl[sp(ls[3])]]
            else:
                arr = amps[name]
            ops.append(arr)
            subs.append(''.join(lab[l] for l in ls))
        res = ''.join(lab[l] for l in ext)
        out += float(coef) * np.einsum(','.join(subs) + '->' + res, *ops, optimize=True)
    return out


def unique_triples(O, V):
    for occ in itertools.combinations(range(O), 3):
        for vir in itertools.combinations(range(V), 3):
            yield occ, vir


# ---------------------------------------------------------------------------
# determinant space
# ---------------------------------------------------------------------------
class ExactCRCC:
    """Exact CR-CC(2,3) quantities for given CCSD amplitudes (dense spin-orbital t1, t2)."""

    def __init__(self, h, v, nocc, t1, t2):
        self.det = DetCC(h, v, nocc)
        self.O = nocc
        self.V = h.shape[0] - nocc
        self.ts = {1: t1, 2: t2}
        d = self.det
        self.E = float(d.phi @ self.hbar(d.phi))

    def hbar(self, vec):
        d = self.det
        return d.exp_t(self.ts, d.apply_h(d.exp_t(self.ts, vec, 1.0)), -1.0)

    def ket(self, occ, vir):
        d = self.det
        base = d.fs.string([(i, False) for i in reversed(occ)], d.phi)
        return d.fs.string([(self.O + a, True) for a in vir], base)

    def space(self, level):
        return [(o, v) for o in itertools.combinations(range(self.O), level)
                for v in itertools.combinations(range(self.V), level)]

    def solve(self):
        d = self.det
        O, V = self.O, self.V
        sd = self.space(1) + self.space(2)
        kets = [self.ket(o, v) for o, v in sd]
        hk = [self.hbar(k) for k in kets]
        n = len(sd)
        A = np.zeros((n, n))
        b = np.zeros(n)
        for mu in range(n):
            b[mu] = d.phi @ hk[mu]
            for nu in range(n):
                A[nu, mu] = kets[nu] @ hk[mu]
        A -= self.E * np.eye(n)
        lam = np.linalg.solve(A.T, -b)
        self.lam = dict(zip(sd, lam))
        # dense antisymmetric lambda tensors
        self.l1 = np.zeros((V, O))
        self.l2 = np.zeros((V, V, O, O))
        for (o, v), x in self.lam.items():
            if len(o) == 1:
                self.l1[v[0], o[0]] = x
            else:
                _fill(self.l2, v, o, x)
        # triples
        trip = self.space(3)
        self.M3, self.L3, self.Dexact = {}, {}, {}
        lk = {k: kets[q] for q, k in enumerate(sd)}
        for o, v in trip:
            k = self.ket(o, v)
            hkk = self.hbar(k)
            self.M3[(o, v)] = float(k @ self.hbar(d.phi))
            self.L3[(o, v)] = float(d.phi @ hkk + sum(self.lam[s] * (lk[s] @ hkk) for s in sd))
            self.Dexact[(o, v)] = self.E - float(k @ hkk)
        self._diag()
        return self

    def _diag(self):
        """One- and two-body Hbar diagonals from 1- and 2-quasiparticle states."""
        d = self.det
        O, V = self.O, self.V
        E = self.E
        ev = lambda x: float(x @ self.hbar(x))
        hole = lambda i, x: d.fs.ann(i, x)
        part = lambda a, x: d.fs.cre(O + a, x)
        self.h1o = np.array([E - ev(hole(i, d.phi)) for i in range(O)])
        self.h1v = np.array([ev(part(a, d.phi)) - E for a in range(V)])
        self.h2oo = np.zeros((O, O))
        for i in range(O):
            for j in range(O):
                if i != j:
                    self.h2oo[i, j] = ev(hole(j, hole(i, d.phi))) - E + self.h1o[i] + self.h1o[j]
        self.h2vv = np.zeros((V, V))
        for a in range(V):
            for b in range(V):
                if a != b:
                    self.h2vv[a, b] = ev(part(b, part(a, d.phi))) - E - self.h1v[a] - self.h1v[b]
        self.h2vo = np.zeros((V, O))
        for a in range(V):
            for i in range(O):
                self.h2vo[a, i] = -(ev(part(a, hole(i, d.phi))) - E - self.h1v[a] + self.h1o[i])

    def denominators(self, occ, vir, fdiag):
        """(D_A, D_B, D_C, D_exact) of one unique triple; fdiag = Fock diagonal (occ, vir)."""
        O = self.O
        da = sum(fdiag[i] for i in occ) - sum(fdiag[O + a] for a in vir)
        db = sum(self.h1o[i] for i in occ) - sum(self.h1v[a] for a in vir)
        dc = db
        for i, j in itertools.combinations(occ, 2):
            dc -= self.h2oo[i, j]
        for a, b in itertools.combinations(vir, 2):
            dc -= self.h2vv[a, b]
        for a in vir:
            for i in occ:
                dc += self.h2vo[a, i]
        return da, db, dc, self.Dexact[(occ, vir)]

    def energies(self, fdiag):
        e = np.zeros(4)
        for key in self.M3:
            lm = self.L3[key] * self.M3[key]
            ds = self.denominators(key[0], key[1], fdiag)
            for q in range(4):
                e[q] += lm / ds[q]
        return e


def _fill(arr, vir, occ, x):
    n = len(vir)
    for pv in itertools.permutations(range(n)):
        for po in itertools.permutations(range(n)):
            s = _perm_sign(pv) * _perm_sign(po)
            arr[tuple(vir[k] for k in pv) + tuple(occ[k] for k in po)] = s * x


# ---------------------------------------------------------------------------
# dense spin-orbital restatement of the reference algorithm
# ---------------------------------------------------------------------------
L_BLOCKS = ('T1A', 'T1B', 'T2A', 'T2B', 'T2C')


class DenseCRCC:
    """CR-CC(2,3) after a converged CCSD (``oracle.densecc.DenseCC`` state ``tvec``)."""

    def __init__(self, cc, tvec, e_cor, shift=0.0, occ_a=None, occ_b=None, bbb_quirk=True):
        self.bbb_quirk = bbb_quirk
        self.cc = cc
        self.so = cc.so
        self.dims = cc.dims
        self.layout = cc.layout
        self.e_cor = e_cor
        self.shift = shift
        d = self.dims
        self.occ_a = d.occ_a if occ_a is None else occ_a
        self.occ_b = d.occ_b if occ_b is None else occ_b
        so = self.so
        blocks = {b: self.layout.view(tvec, b) for b in L_BLOCKS}
        ts = so.from_blocks(blocks, 2)
        self.t1, self.t2 = ts[1], ts[2]
        self.fd, self.vd = so.dressed(self.t1)
        self._hbar_diag()

    # -- Hbar(CCSD) diagonals ---------------------------------------------------
    def _hbar_diag(self):
        so = self.so
        O, N = so.O, so.N
        fd, vd, t2 = self.fd, self.vd, self.t2
        o, v = slice(0, O), slice(O, N)
        v_oovv = self.so.v[o, o, v, v]
        # h(i,i) = f~(i,i) + 1/2 sum_{m e f} <im||ef> t(ef,im)
        self.h1o = np.diag(fd[o, o]) + 0.5 * np.einsum('imef,efim->i', v_oovv, t2)
        # h(a,a) = f~(a,a) - 1/2 sum_{m n f} <mn||af> t(af,mn)
        self.h1v = np.diag(fd[v, v]) - 0.5 * np.einsum('mnaf,afmn->a', v_oovv, t2)
        # two-body diagonals: [i,j,i,j], [a,b,a,b], [a,i,a,i]
        self.h2oo = np.einsum('ijij->ij', vd[o, o, o, o]) + 0.5 * np.einsum('ijef,efij->ij', v_oovv, t2)
        self.h2vv = np.einsum('abab->ab', vd[v, v, v, v]) + 0.5 * np.einsum('mnab,abmn->ab', v_oovv, t2)
        self.h2vo = np.einsum('aiai->ai', vd[v, o, v, o]) - np.einsum('inaf,afin->ai', v_oovv, t2)
        # three-body pieces (cal_d3): w1[x, p, q] = sum_e <pq||xe> t(xe,pq);
        # w2[x, z, y] = sum_m <ym||xz> t(xz,ym)
        spin = so.spin
        sv = spin[O:]
        keep = np.ones(so.V, dtype=bool)
        # beta virtuals with absolute index below occ_a + 2 (relative index <= occ_a - occ_b)
        vb_rel = np.cumsum(sv == 1) - 1
        drop = (sv == 1) & (vb_rel <= self.occ_a - self.occ_b)
        if self.bbb_quirk:
            keep[drop] = False
        self.w1 = np.einsum('pqxe,xepq->xpq', v_oovv, t2)
        self.w1_bbb = np.einsum('pqxe,xepq->xpq', v_oovv[:, :, :, keep], t2[:, keep])
        self.w2 = np.einsum('ymxz,xzym->xzy', v_oovv, t2)

    def hbar_fdiag(self):
        """Full-range (occ, vir) spin-orbital Hbar one-body diagonal."""
        return np.concatenate([self.h1o, self.h1v])

    # -- left CCSD --------------------------------------------------------------
    def _to_dense_l(self, lvec):
        blocks = {b: self.layout.view(lvec, b) for b in L_BLOCKS}
        ls = self.so.from_blocks(blocks, 2)
        return ls[1], ls[2]

    def left_residual(self, l1, l2):
        so = self.so
        amps = {'t1': self.t1, 't2': self.t2, 'l1': l1, 'l2': l2}
        r1 = eval_terms(lagrange.left_residual_terms(1), 1, amps, so.f, so.v, so.O)
        r2 = eval_terms(lagrange.left_residual_terms(2), 2, amps, so.f, so.v, so.O)
        return r1, r2

    def _spin_diag(self):
        """Hbar one-body diagonal per spin in the (occ, vir) orbital order of a block."""
        so = self.so
        spin = so.spin
        O = so.O
        ha = np.concatenate([self.h1o[spin[:O] == 0], self.h1v[spin[O:] == 0]])
        hb = np.concatenate([self.h1o[spin[:O] == 1], self.h1v[spin[O:] == 1]])
        return ha, hb

    def update(self, lvec):
        """update_l2 + left_jacobi_update: all residuals from the old lambda, then Jacobi."""
        l1, l2 = self._to_dense_l(lvec)
        r1, r2 = self.left_residual(l1, l2)
        rb = self.so.to_blocks({1: r1, 2: r2}, list(L_BLOCKS))
        self.lh_norm = float(sum(np.sum(rb[b] ** 2) for b in L_BLOCKS))
        ha, hb = self._spin_diag()
        for b in L_BLOCKS:
            lv = self.layout.view(lvec, b)
            D = S.denominator(b, lv.shape, ha, hb, self.dims, self.shift - self.e_cor)
            lv[...] = S.jacobi_block(b, lv.copy(), rb[b], D)

    def energy(self, lvec):
        return float(np.sqrt(self.lh_norm)) + self.e_cor

    def solve_left(self, diis_space=5, max_iter=60, tol=1e-8):
        lvec = np.zeros(self.layout.t_size)
        vs = self.layout.vec_size('CCSD')
        e, it, failed, hist = S.jacobi_iter(self.update, self.energy, lvec, vs, diis_space, max_iter, tol)
        self.lvec = lvec
        self.l1, self.l2 = self._to_dense_l(lvec)
        return e, it, failed, hist

    # -- triples ---------------------------------------------------------------
    def moments(self):
        amps = {'t2': self.t2}
        return eval_terms(lagrange.triples_moment_terms(), 3, amps, self.fd, self.vd, self.so.O)

    def left_projections(self):
        amps = {'t2': self.t2, 'l1': self.l1, 'l2': self.l2}
        return eval_terms(lagrange.triples_left_terms(), 3, amps, self.fd, self.vd, self.so.O)

    def denominators(self, occ, vir):
        so = self.so
        O = so.O
        spin = so.spin
        f = np.diag(so.f)
        da = sum(f[i] for i in occ) - sum(f[O + a] for a in vir)
        db = sum(self.h1o[i] for i in occ) - sum(self.h1v[a] for a in vir)
        dc = db
        for i, j in itertools.combinations(occ, 2):
            dc -= self.h2oo[i, j]
        for a, b in itertools.combinations(vir, 2):
            dc -= self.h2vv[a, b]
        for a in vir:
            for i in occ:
                dc += self.h2vo[a, i]
        dd = dc
        for x in vir:
            for p, q in itertools.combinations(occ, 2):
                allb = spin[O + x] == 1 and spin[p] == 1 and spin[q] == 1
                dd += (self.w1_bbb if allb else self.w1)[x, p, q]
        for x, z in itertools.combinations(vir, 2):
            for y in occ:
                dd += self.w2[x, z, y]
        return da, db, dc, dd

    def energies(self, active=None):
        """The four corrections; ``active = (act_occ_b, act_unocc_a)`` (CC(t;3)) leaves out the
        triples with an occupied spatial orbital above act_occ_b and a virtual one up to
        act_unocc_a (``src/mm_correct.f90:61-62,131``)."""
        M = self.moments()
        L = self.left_projections()
        self.M3, self.L3 = M, L
        so = self.so
        O, V = so.O, so.V
        spin = so.spin
        e = np.zeros(4)
        for occ, vir in unique_triples(O, V):
            if sorted(spin[list(occ)]) != sorted(spin[[O + a for a in vir]]):
                continue
            if active is not None:
                froz = self.dims.froz
                top = max(so.sp[i][0] for i in occ) + froz + 1        # 1-based spatial orbitals
                low = min(so.sp[O + a][0] for a in vir) + froz + 1
                if top > active[0] and low <= active[1]:
                    continue
            lm = L[vir + occ] * M[vir + occ]
            ds = self.denominators(occ, vir)
            for q in range(4):
                e[q] += lm / ds[q]
        return e
