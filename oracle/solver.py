"""CPU restatement of ccq's iteration driver (test infrastructure only).

  * ``jacobi_iter``     <- ``jacobi_iter`` (``src/solve_cc.f90:175-269``) and
                           ``check_convergence`` (``:293-316``)
  * ``Ring``/``diis``   <- ``write_vecs``/``read_vec``/``residuum``/``calc_diis``/
                           ``construct_b_mat`` (``src/diis.F90:11-349``)
  * ``jacobi_block``    <- the Jacobi steps at the end of every ``t*_update``
                           (e.g. ``src/cc/t1A_update.f90:518-525``,
                           ``src/cc/t2A_update.f90:1885-1901``,
                           ``src/cc/t3A_update.f90:2566-2620``)
  * ``tran3bto3c``      <- ``src/cc/tran3Bto3C.f90:1-31``
  * ``BLOCK_ORDER``     <- ``update_clusters_t4`` (``src/update_cc.F90:12-323``)

Quirks kept on purpose: DIIS runs every ``diis_space+1`` iterations and
extrapolates with the OLDEST ``diis_space`` vectors of the ring; the bordered
B matrix has -1 in its corner; the printed residuum is sqrt(||dt||); three
consecutive |dE| < tol are needed.  Only ``tests/`` and ``bench.py``'s CPU
baseline use this module.
"""
from __future__ import annotations

import itertools

import numpy as np

BLOCK_ORDER = ['T2A', 'T2C', 'T2B', 'T1A', 'T1B', 'T3A', 'T3D', 'T3B', 'T3C',
               'T4A', 'T4B', 'T4C', 'T4D', 'T4E']
RHF_COPY = {'T2C': 'T2A', 'T1B': 'T1A', 'T3D': 'T3A', 'T3C': 'tran3bto3c', 'T4D': 'tran4bto4d', 'T4E': 'T4A'}


def block_spins(name):
    n = int(name[1])
    nb = 'ABCDE'.index(name[2])
    return [0] * (n - nb) + [1] * nb


def _runs(spins):
    out = []
    start = 0
    for k in range(1, len(spins) + 1):
        if k == len(spins) or spins[k] != spins[start]:
            out.append(list(range(start, k)))
            start = k
    return out


def canonical_mask(name, shape):
    """True where indices increase strictly within each same-spin run."""
    n = int(name[1])
    spins = block_spins(name)
    grids = np.indices(shape, sparse=True)
    mask = np.ones(shape, dtype=bool)
    for part in (0, n):
        for run in _runs(spins):
            for a, b in zip(run[:-1], run[1:]):
                mask &= grids[part + a] < grids[part + b]
    return mask


def antisym_fill(name, t):
    """Rebuild a block from its canonical elements (all sign-permuted copies)."""
    n = int(name[1])
    spins = block_spins(name)
    runs = _runs(spins)
    canon = np.where(canonical_mask(name, t.shape), t, 0.0)
    out = np.zeros_like(t)
    perms_part = []
    for run in runs:
        perms_part.append(list(itertools.permutations(run)))
    for po in itertools.product(*perms_part):
        for pv in itertools.product(*perms_part):
            so = 1
            axes = list(range(2 * n))
            for run, p in zip(runs, po):
                so *= _psign([run.index(x) for x in p])
                for src, dst in zip(run, p):
                    axes[dst] = src
            sv = 1
            for run, p in zip(runs, pv):
                sv *= _psign([run.index(x) for x in p])
                for src, dst in zip(run, p):
                    axes[n + dst] = n + src
            out += so * sv * canon.transpose(axes)
    return out


def _psign(p):
    s = 1
    for i in range(len(p)):
        for j in range(i + 1, len(p)):
            if p[j] < p[i]:
                s = -s
    return s


def denominator(name, shape, fdiag_a, fdiag_b, dims, shift):
    """f_aa + f_bb + .. - f_ii - .. + shift in block index order (occ.., vir..)."""
    n = int(name[1])
    spins = block_spins(name)
    D = np.full(shape, shift)
    for k, s in enumerate(spins):
        fd = fdiag_a if s == 0 else fdiag_b
        o = dims.oa if s == 0 else dims.ob
        eo = fd[:o]
        ev = fd[o:]
        shp = [1] * (2 * n)
        shp[k] = len(eo)
        D = D - eo.reshape(shp)
        shp = [1] * (2 * n)
        shp[n + k] = len(ev)
        D = D + ev.reshape(shp)
    return D


def jacobi_block(name, t, R, D):
    """t <- t - R/D on canonical elements, then antisymmetric fill."""
    mask = canonical_mask(name, t.shape)
    new = np.where(mask, t - R / D, 0.0)
    return antisym_fill(name, new)


def tran3bto3c(t3b):
    """T3C[i,j,k,a,b,c] = T3B[j,k,i,b,c,a] on j<k, b<c, then fill."""
    t3c = t3b.transpose(2, 0, 1, 5, 3, 4).copy()
    return antisym_fill('T3C', np.where(canonical_mask('T3C', t3c.shape), t3c, 0.0))


def tran4bto4d(t4b):
    """Closed-shell spin flip of T4B (alpha^3 beta) into T4D (alpha beta^3)."""
    # T4D[i,j,k,l,a,b,c,d] (a: alpha; b,c,d: beta) = T4B with spins flipped,
    # reordered alpha-first: occ (j,k,l,i), vir (b,c,d,a) -> cyclic, sign -1 each
    t4d = t4b.transpose(3, 0, 1, 2, 7, 4, 5, 6).copy()
    return antisym_fill('T4D', np.where(canonical_mask('T4D', t4d.shape), t4d, 0.0))


class Ring:
    """HBM/CPU stand-in for the ``cc_iter_mat-<k>.bin`` files."""

    def __init__(self, ds, size):
        self.ds = ds
        self.slots = [None] * (ds + 1)
        self.size = size

    def slot(self, it):
        s = it % (self.ds + 1)
        return self.ds + 1 if s == 0 else s

    def write(self, it, vec):
        self.slots[self.slot(it) - 1] = vec[:self.size].copy()

    def read(self, it):
        return self.slots[self.slot(it) - 1]

    def residuum(self, it):
        v1 = np.zeros(self.size) if it == 1 else self.read(it - 1)
        v2 = self.read(it)
        d = v1 - v2
        return float(np.sqrt(np.sqrt(d @ d)))

    def diis(self):
        ds = self.ds
        B = np.zeros((ds + 1, ds + 1))
        for i in range(1, ds + 1):
            v3 = self.read(i + 1) - self.read(i)
            for j in range(i, ds + 1):
                v2 = self.read(j + 1) - self.read(j)
                B[i - 1, j - 1] += v3 @ v2
        for i in range(ds):
            for j in range(i + 1, ds):
                B[j, i] = B[i, j]
        B[:, ds] = -1.0
        B[ds, :] = -1.0
        C = np.zeros(ds + 1)
        C[ds] = -1.0
        c = np.linalg.solve(B, C)
        out = np.zeros(self.size)
        for i in range(1, ds + 1):
            out += c[i - 1] * self.read(i)
        return out


def jacobi_iter(update, energy, tvec, vec_size, diis_space=5, max_iter=60, tol=1e-4, log=None, pack=None,
                unpack=None):
    """Fixed-point loop of ccq.  ``update(tvec)`` updates in place.

    ``pack(tvec)`` / ``unpack(vec)`` (optional) map the T vector to the DIIS vector and back: for
    active-space CCSDt, ccq's t_vec is the compressed one of get_t_sizes_act
    (src/utils/cc_utils.f90:560-630), over which its ring, residuum and extrapolation run.
    Returns (e_cor, iterations, failed, history[(e, de, res)]).
    """
    conv = [1.0, 1.0, 1.0]
    en_cor = 0.0
    ring = Ring(diis_space, vec_size)
    hist = []
    failed = False
    it = 0
    for it in range(1, max_iter + 1):
        update(tvec)
        e_new = energy(tvec)
        diff = en_cor - e_new
        conv = [conv[1], conv[2], diff]
        en_cor = e_new
        ring.write(it, tvec if pack is None else pack(tvec))
        res = ring.residuum(it)
        if it % (diis_space + 1) == 0:
            if unpack is None:
                tvec[:vec_size] = ring.diis()
            else:
                tvec[:] = unpack(ring.diis())
        hist.append((e_new, diff, res))
        if log:
            log(f"  {it:4d}{e_new:15.10f}{diff:15.10f}{res:15.10f}")
        if all(abs(c) < tol for c in conv):
            break
        if np.isnan(e_new):
            failed = True
            break
        if it == max_iter:
            failed = True
    return en_cor, it, failed, hist
