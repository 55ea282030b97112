"""Dense spin-orbital CC oracle (test infrastructure only).

Evaluates the symbolic spin-orbital residuals of ``ccq_b200.eqgen.wick`` with
``numpy.einsum`` on dense spin-orbital tensors, with no spin integration, so it
checks the spin-block plan compiler independently.  It restates the
reference's algorithm (``src/update_cc.F90:12-323`` block order with in-place
updates, the Jacobi step of ``src/cc/t2A_update.f90:1885-1901``) on small
systems; the spin-blocked numpy executor in ``oracle/blockcc.py`` covers the
large ones.

Spin-orbital order: occupied alpha, occupied beta, virtual alpha, virtual beta.
Only ``tests/`` use this module.
"""
from __future__ import annotations

import numpy as np

from ccq_b200.eqgen import wick

LETTERS = 'abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ'


class SpinOrbitalSystem:
    """Dense spin-orbital h (core), v (antisymmetrised), f from spin blocks."""

    def __init__(self, f_a, f_b, v_aa, v_ab, v_bb, oa, ob):
        n = v_aa.shape[0]
        self.n, self.oa, self.ob = n, oa, ob
        self.va, self.vb = n - oa, n - ob
        self.O = oa + ob
        self.V = self.va + self.vb
        self.N = self.O + self.V
        sp = []   # (spatial index in active range, spin 0/1)
        sp += [(k, 0) for k in range(oa)]
        sp += [(k, 1) for k in range(ob)]
        sp += [(oa + k, 0) for k in range(self.va)]
        sp += [(ob + k, 1) for k in range(self.vb)]
        self.sp = sp
        x = np.array([s[0] for s in sp])
        s = np.array([s[1] for s in sp])
        self.spin = s
        N = self.N
        # core h from the Fock blocks: h = f - sum_occ v
        h_a = f_a - np.einsum('piqi->pq', v_aa[:, :oa, :, :oa]) - np.einsum('piqi->pq', v_ab[:, :ob, :, :ob])
        h_b = f_b - np.einsum('piqi->pq', v_bb[:, :ob, :, :ob]) - np.einsum('ipiq->pq', v_ab[:oa, :, :oa, :])
        h = np.zeros((N, N))
        f = np.zeros((N, N))
        for P in range(N):
            for Q in range(N):
                if s[P] == s[Q]:
                    hb = h_a if s[P] == 0 else h_b
                    fb = f_a if s[P] == 0 else f_b
                    h[P, Q] = hb[x[P], x[Q]]
                    f[P, Q] = fb[x[P], x[Q]]
        v = np.zeros((N, N, N, N))
        X = np.ix_(x, x, x, x)
        vaa = v_aa[X]
        vbb = v_bb[X]
        S0 = s[:, None, None, None]
        S1 = s[None, :, None, None]
        S2 = s[None, None, :, None]
        S3 = s[None, None, None, :]
        aaaa = (S0 == 0) & (S1 == 0) & (S2 == 0) & (S3 == 0)
        bbbb = (S0 == 1) & (S1 == 1) & (S2 == 1) & (S3 == 1)
        v[aaaa] = vaa[aaaa]
        v[bbbb] = vbb[bbbb]
        # mixed: <pq|rs> with p,r same spin and q,s same spin
        vab_pqrs = v_ab[np.ix_(x, x, x, x)]                       # v_ab[xp,xq,xr,xs]
        vab_qpsr = v_ab[np.ix_(x, x, x, x)].transpose(1, 0, 3, 2)  # v_ab[xq,xp,xs,xr]
        vab_pqsr = v_ab[np.ix_(x, x, x, x)].transpose(0, 1, 3, 2)  # v_ab[xp,xq,xs,xr]
        vab_qprs = v_ab[np.ix_(x, x, x, x)].transpose(1, 0, 2, 3)  # v_ab[xq,xp,xr,xs]
        m = (S0 == 0) & (S1 == 1) & (S2 == 0) & (S3 == 1)
        v[m] = vab_pqrs[m]
        m = (S0 == 1) & (S1 == 0) & (S2 == 1) & (S3 == 0)
        v[m] = vab_qpsr[m]
        m = (S0 == 0) & (S1 == 1) & (S2 == 1) & (S3 == 0)
        v[m] = -vab_pqsr[m]
        m = (S0 == 1) & (S1 == 0) & (S2 == 0) & (S3 == 1)
        v[m] = -vab_qprs[m]
        self.h, self.f, self.v = h, f, v

    # --- amplitude conversion -------------------------------------------------
    def occ_idx(self, spin):
        return list(range(self.oa)) if spin == 0 else list(range(self.oa, self.O))

    def vir_idx(self, spin):
        return list(range(self.va)) if spin == 0 else list(range(self.va, self.V))

    def from_blocks(self, blocks, nmax):
        """Dense antisymmetric t_n[a.., i..] from spin blocks (TLayout order)."""
        ts = {}
        for n in range(1, nmax + 1):
            ts[n] = np.zeros((self.V,) * n + (self.O,) * n)
        for name, arr in blocks.items():
            n = int(name[1])
            nb = 'ABCDE'.index(name[2])   # number of beta electrons
            spins = [0] * (n - nb) + [1] * nb
            oi = [self.occ_idx(sp) for sp in spins]
            vi = [self.vir_idx(sp) for sp in spins]
            # arr axes: occ slots then vir slots
            grid = np.ix_(*(vi + oi))
            val = arr.transpose(list(range(n, 2 * n)) + list(range(n)))
            _fill_antisym(ts[n], grid, val, n)
        return ts

    def to_blocks(self, ts, names):
        out = {}
        for name in names:
            n = int(name[1])
            nb = 'ABCDE'.index(name[2])
            spins = [0] * (n - nb) + [1] * nb
            oi = [self.occ_idx(sp) for sp in spins]
            vi = [self.vir_idx(sp) for sp in spins]
            sub = ts[n][np.ix_(*(vi + oi))]
            out[name] = np.ascontiguousarray(sub.transpose(list(range(n, 2 * n)) + list(range(n))))
        return out

    # --- dressed Hamiltonian --------------------------------------------------
    def dressed(self, t1):
        """f, v of exp(-T1) H exp(T1) (t1[a,i])."""
        O, N = self.O, self.N
        A = np.eye(N)
        B = np.eye(N)
        A[:O, O:] = -t1.T
        B[O:, :O] = t1
        hd = A.T @ self.h @ B
        vd = np.einsum('pP,qQ,pqrs,rR,sS->PQRS', A, A, self.v, B, B, optimize=True)
        fd = hd + np.einsum('piqi->pq', vd[:, :O, :, :O])
        return fd, vd

    def residual(self, ts, level, tranks):
        """R[a.., i..] for excitation ``level`` with the generated equations."""
        fd, vd = self.dressed(ts[1])
        O = self.O
        sl = {'o': slice(0, O), 'v': slice(O, self.N)}
        terms = wick.residual_terms(level, tuple(tranks))
        ext = wick.ext_labels(level)
        R = np.zeros((self.V,) * level + (self.O,) * level)
        for coef, tensors in terms:
            ops = []
            subs = []
            lab = {}
            for name, ls in tensors:
                for l in ls:
                    if l not in lab:
                        lab[l] = LETTERS[len(lab)]
                sub = ''.join(lab[l] for l in ls)
                if name == 'f':
                    arr = fd[sl[_sp(ls[0])], sl[_sp(ls[1])]]
                elif name == 'v':
                    arr = vd[sl[_sp(ls[0])], sl[_sp(ls[1])], sl[_sp(ls[2])], sl[_sp(ls[3])]]
                else:
                    arr = ts[int(name[1])]
                ops.append(arr)
                subs.append(sub)
            out = ''.join(lab[l] for l in ext)
            R += float(coef) * np.einsum(','.join(subs) + '->' + out, *ops, optimize=True)
        return R

    def energy(self, ts):
        t1 = ts[1]
        t2 = ts[2]
        O = self.O
        f_ov = self.f[:O, O:]
        v_oovv = self.v[:O, :O, O:, O:]
        e = np.einsum('ia,ai->', f_ov, t1)
        e += 0.25 * np.einsum('ijab,abij->', v_oovv, t2)
        e += 0.5 * np.einsum('ijab,ai,bj->', v_oovv, t1, t1)
        return float(e)

    def denominators(self, level, shift=0.0):
        eo = np.diag(self.f)[:self.O]
        ev = np.diag(self.f)[self.O:]
        D = np.zeros((self.V,) * level + (self.O,) * level)
        for k in range(level):
            shp = [1] * (2 * level)
            shp[k] = self.V
            D = D + ev.reshape(shp)
            shp = [1] * (2 * level)
            shp[level + k] = self.O
            D = D - eo.reshape(shp)
        return D + shift


def _sp(l):
    return 'o' if l[0] in 'io' else 'v'


def _fill_antisym(dst, grid, val, n):
    """Write val at grid and every antisymmetric permutation of its slots."""
    import itertools
    vi = [np.asarray(g).reshape(-1) for g in grid[:n]]
    oi = [np.asarray(g).reshape(-1) for g in grid[n:]]
    for pv in itertools.permutations(range(n)):
        sv = _psign(pv)
        for po in itertools.permutations(range(n)):
            so = _psign(po)
            idx = [vi[k] for k in pv] + [oi[k] for k in po]
            dst[np.ix_(*idx)] = sv * so * val.transpose(list(pv) + [n + k for k in po])


def _psign(p):
    s = 1
    p = list(p)
    for i in range(len(p)):
        for j in range(i + 1, len(p)):
            if p[j] < p[i]:
                s = -s
    return s
