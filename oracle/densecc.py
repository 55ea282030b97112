"""Small-system CC oracle: dense spin-orbital residuals + ccq's driver.

Composes ``oracle.spinorb`` (residuals from the symbolic equations, no spin
integration) with ``oracle.solver`` (ccq's in-place block sweep, Jacobi step,
DIIS and convergence rule).  Only ``tests/`` use this module.
"""
from __future__ import annotations

import numpy as np

from ccq_b200 import integrals as I
from oracle import solver as S
from oracle.spinorb import SpinOrbitalSystem

METHOD = {'CCSD': (2,), 'CCSDT': (2, 3), 'CCSDTQ': (2, 3, 4)}


def active_mask(name, shape, dims, active):
    """CCSDt triples kept: >= 1 active occupied and >= 1 active virtual index.

    ``active = (act_occ_b, act_unocc_a)``: ccq's boundaries (``src/parser.f90:495-499``,
    ``src/update_cc.F90:412-440``): occupied spatial orbitals above act_occ_b and
    virtual ones up to act_unocc_a are active, for both spins.
    """
    m1, m2 = active
    nb = 'ABCD'.index(name[2])
    spins = [0] * (3 - nb) + [1] * nb
    occ_any = np.zeros(shape, dtype=bool)
    vir_any = np.zeros(shape, dtype=bool)
    for d in range(3):
        idx = np.arange(shape[d]).reshape([-1 if e == d else 1 for e in range(6)])
        occ_any |= np.broadcast_to(idx >= m1 - dims.froz, shape)
    for d in range(3):
        occ = dims.occ_a if spins[d] == 0 else dims.occ_b
        idx = np.arange(shape[3 + d]).reshape([-1 if e == 3 + d else 1 for e in range(6)])
        vir_any |= np.broadcast_to(idx < m2 - occ, shape)
    return occ_any & vir_any


class DenseCC:
    def __init__(self, f_a, f_b, v_aa, v_ab, v_bb, dims: I.Dims, method, shift=0.0, rhf=False, active=None,
                 external=False):
        self.active = active   # CCSDt: (act_occ_b, act_unocc_a), triples outside the active space held at zero
        # externally corrected CC: T3 / T4 stay as given, only T1 and T2 are updated, DIIS over T1 + T2
        self.external = external
        self.dims = dims
        self.method = method
        self.tranks = METHOD[method]
        self.nmax = max(self.tranks)
        self.shift = shift
        self.rhf = rhf
        fr = dims.froz
        self.fa = f_a[fr:, fr:]
        self.fb = f_b[fr:, fr:]
        self.so = SpinOrbitalSystem(self.fa, self.fb, v_aa, v_ab, v_bb, dims.oa, dims.ob)
        self.layout = I.TLayout(dims)
        self.t4 = {b: np.zeros(s) for b, s in self.layout.t4_shape.items()} if self.nmax >= 4 else {}
        self.blocks = [b for b in S.BLOCK_ORDER if int(b[1]) <= (2 if external else self.nmax)]

    def _blocks(self, tvec):
        out = {b: self.layout.view(tvec, b) for b in I.T_VEC_ORDER if int(b[1]) <= self.nmax}
        out.update(self.t4)
        return out

    def update(self, tvec):
        fda = np.diag(self.fa)
        fdb = np.diag(self.fb)
        for name in self.blocks:
            blocks = self._blocks(tvec)
            if self.rhf and name in S.RHF_COPY:
                src = S.RHF_COPY[name]
                if src == 'tran3bto3c':
                    new = S.tran3bto3c(blocks['T3B'])
                elif src == 'tran4bto4d':
                    new = S.tran4bto4d(blocks['T4B'])
                else:
                    new = blocks[src].copy()
            else:
                ts = self.so.from_blocks(blocks, self.nmax)
                level = int(name[1])
                R = self.so.residual(ts, level, self.tranks)
                Rb = self.so.to_blocks({level: R}, [name])[name]
                D = S.denominator(name, blocks[name].shape, fda, fdb, self.dims, self.shift)
                new = S.jacobi_block(name, blocks[name], Rb, D)
                if self.active is not None and level == 3:
                    new = np.where(active_mask(name, new.shape, self.dims, self.active), new, 0.0)
            if name in self.t4:
                self.t4[name] = new
            else:
                self.layout.view(tvec, name)[...] = new

    def energy(self, tvec):
        blocks = self._blocks(tvec)
        ts = self.so.from_blocks({k: v for k, v in blocks.items() if int(k[1]) <= 2}, 2)
        return self.so.energy(ts)

    def solve(self, diis_space=5, max_iter=60, tol=1e-8, log=None, t0=None, compressed_diis=False):
        """compressed_diis (with an active space): DIIS over ccq's compressed CCSDt T vector, as ccq runs
        CCSDt (its t_vec is get_t_sizes_act's)."""
        tvec = np.zeros(self.layout.t_size) if t0 is None else np.array(t0, dtype=np.float64)
        vs = self.layout.vec_size('CCSD' if self.external else self.method)
        pack = unpack = None
        if compressed_diis:
            from oracle import ccsdt_layout as CL
            d = self.dims
            dims = (d.froz, d.occ_a, d.occ_b, d.orbs)
            m1, m2 = self.active
            pack = lambda t: CL.compress(t, dims, m1, m2)  # noqa: E731
            unpack = lambda v: CL.expand(v, dims, m1, m2)  # noqa: E731
            vs = CL.pos_offsets(*dims, m1, m2)[-1] - 1
        e, it, failed, hist = S.jacobi_iter(self.update, self.energy, tvec, vs, diis_space, max_iter, tol, log,
                                            pack, unpack)
        return e, it, failed, hist, tvec
