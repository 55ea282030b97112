"""Integral files, spin blocks, Fock operator and the T-vector layout of ccq.

Mirrors the reference's input side so that a ccq input deck runs unchanged:
  * ``read_onebody``   <- ``load_e1int``  (``src/integrals.f90:11-43``)
  * ``read_twobody``   <- ``load_e2int``  (``src/integrals.f90:45-91``)
  * ``read_fcidump``   <- ``load_fcidump`` (``src/integrals.f90:93-210``), through
    the library's native reader (``ccq_b200_fcidump_read``)
  * ``spin_blocks``    <- ``load_ints``   (``src/integrals.f90:212-297``)
  * ``fock``           <- ``gen_fock_operator`` (``src/integrals.f90:300-364``)
  * ``hf_energy``      <- ``calc_hf_energy`` (``src/energy.f90:49-101``)
  * ``TLayout``        <- ``get_t_sizes`` (``src/utils/cc_utils.f90:479-559``)

Array conventions.  Python arrays are C-ordered with the reference's index
meaning: ``e2int[i, j, a, b] = <ij|ab>`` (physicist), ``v_aa[p, q, r, s] =
<pq||rs>``, ``v_ab[p, q, r, s] = <p_a q_b | r_a s_b>``.  Amplitude blocks use
the memory order of the reference's Fortran arrays, read in C order:
``t2a(b,a,j,i)`` (Fortran) is ``T2A[i, j, a, b]`` here, so the flat T vector is
byte-identical to ccq's ``t_vec``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def count_lines(path):
    with open(path) as fh:
        return sum(1 for _ in fh)


def read_onebody(path, orbs):
    """``value index`` lines, i = 1..orbs, j = 1..i (lower triangle, row-major)."""
    n_lines = count_lines(path)
    norb = int(-(1 - math.sqrt(1 + 8 * n_lines)) / 2)
    if norb != orbs:
        raise ValueError("Number of orbitals doesn't match the number of integrals")
    vals = []
    with open(path) as fh:
        for line in fh:
            parts = line.split()
            if not parts:
                continue
            vals.append(float(parts[0].replace('D', 'E').replace('d', 'e')))
    e1 = np.zeros((orbs, orbs))
    k = 0
    for i in range(orbs):
        for j in range(i + 1):
            e1[i, j] = vals[k]
            e1[j, i] = vals[k]
            k += 1
    return e1


def read_twobody(path, orbs):
    """Lines ``i a j b (ia|jb)``; stored as ``e2int[i,j,a,b]``; ``0 0 0 0 E_nuc`` ends.

    As in the reference no permutational symmetry is applied on read: the file
    must list every nonzero permutation.
    """
    e2 = np.zeros((orbs, orbs, orbs, orbs))
    en_repul = 0.0
    raw = np.loadtxt(path, ndmin=2)
    idx = raw[:, :4].astype(np.int64)
    vals = raw[:, 4]
    term = np.where(idx.sum(axis=1) == 0)[0]
    if len(term):
        en_repul = float(vals[term[0]])
        idx = idx[:term[0]]
        vals = vals[:term[0]]
    i, a, j, b = idx[:, 0] - 1, idx[:, 1] - 1, idx[:, 2] - 1, idx[:, 3] - 1
    e2[i, j, a, b] = vals
    return e2, en_repul


def read_fcidump(path, orbs):
    """(e1int, e2int, E_nuc) from the unique integrals of a FCIDUMP file.

    Orbitals are renumbered by ascending orbital energy and every (ia|jb) is
    expanded to its eight permutations, as ``load_fcidump`` does.
    """
    from . import lib
    return lib.fcidump_read(path, orbs)


def write_fcidump(path, e1, e2, en_repul=0.0, nelec=0, eps=None, order=None, thresh=0.0):
    """FCIDUMP with the unique integrals (i >= a, j >= b, (ia) >= (jb)) of e1int/e2int.

    ``order`` relabels orbital p as ``order[p] + 1`` in the file (the reader
    undoes it through the orbital-energy records ``eps``).
    """
    n = e1.shape[0]
    lab = (np.arange(n) if order is None else np.asarray(order)) + 1
    lines = [f" &FCI NORB={n:3d},NELEC={nelec:3d},MS2=0,", "  ORBSYM=" + ",".join("1" * n) + ",", "  ISYM=1,",
             " &END"]
    for i in range(n):
        for a in range(i + 1):
            for j in range(n):
                for b in range(j + 1):
                    if i * (i + 1) // 2 + a < j * (j + 1) // 2 + b:
                        continue
                    v = e2[i, j, a, b]
                    if abs(v) > thresh:
                        lines.append(f"{v: .16E} {lab[i]:4d} {lab[a]:4d} {lab[j]:4d} {lab[b]:4d}")
    for i in range(n):
        for a in range(i + 1):
            if abs(e1[i, a]) > thresh:
                lines.append(f"{e1[i, a]: .16E} {lab[i]:4d} {lab[a]:4d}    0    0")
    if eps is not None:
        for i in range(n):
            lines.append(f"{eps[i]: .16E} {lab[i]:4d}    0    0    0")
    lines.append(f"{en_repul: .16E}    0    0    0    0")
    with open(path, 'w') as fh:
        fh.write("\n".join(lines) + "\n")


def write_onebody(path, e1):
    n = e1.shape[0]
    with open(path, 'w') as fh:
        k = 1
        for i in range(n):
            for j in range(i + 1):
                fh.write(f"{e1[i, j]: .16E} {k:4d}\n")
                k += 1


def write_twobody(path, e2, en_repul=0.0):
    """Writes all n^4 entries as ``i a j b (ia|jb)`` from ``e2int[i,j,a,b]``."""
    n = e2.shape[0]
    ii, aa, jj, bb = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), np.arange(n), indexing='ij')
    vals = e2[ii, jj, aa, bb]
    data = np.stack([ii.ravel() + 1, aa.ravel() + 1, jj.ravel() + 1, bb.ravel() + 1], axis=1)
    with open(path, 'w') as fh:
        lines = [f"{p:5d}{q:5d}{r:5d}{s:5d} {v: .16E}\n" for (p, q, r, s), v in zip(data.tolist(), vals.ravel().tolist())]
        fh.writelines(lines)
        fh.write(f"{0:5d}{0:5d}{0:5d}{0:5d} {en_repul: .16E}\n")


def spin_blocks(e2, froz):
    """Antisymmetrised spin blocks over the active range ``froz..orbs-1``."""
    e = e2[froz:, froz:, froz:, froz:]
    v_ab = e.copy()
    v_aa = e - e.transpose(0, 1, 3, 2)
    return v_aa, v_ab, v_aa.copy()


def fock(e1, e2, occ_a, occ_b):
    """f_a, f_b over the full orbital range, occupied sums include frozen core."""
    f_a = e1.copy()
    f_b = e1.copy()
    ea = e2[:, :occ_a, :, :occ_a]
    eb = e2[:, :occ_b, :, :occ_b]
    coul_a = np.einsum('ikjk->ij', ea)
    exch_a = np.einsum('ikkj->ij', e2[:, :occ_a, :occ_a, :])
    coul_b = np.einsum('ikjk->ij', eb)
    exch_b = np.einsum('ikkj->ij', e2[:, :occ_b, :occ_b, :])
    f_a = f_a + coul_b + (coul_a - exch_a)
    f_b = f_b + coul_a + (coul_b - exch_b)
    # reference fills the lower triangle and mirrors it
    f_a = np.tril(f_a) + np.tril(f_a, -1).T
    f_b = np.tril(f_b) + np.tril(f_b, -1).T
    return f_a, f_b


def hf_energy(e1, e2, occ_a, occ_b):
    e = 0.0
    e += sum(e1[i, i] for i in range(occ_a))
    e += sum(e1[i, i] for i in range(occ_b))
    for i in range(occ_a):
        for j in range(occ_b):
            e += e2[i, j, i, j]
    for i in range(occ_a):
        for j in range(occ_a):
            e += 0.5 * (e2[i, j, i, j] - e2[i, j, j, i])
    for i in range(occ_b):
        for j in range(occ_b):
            e += 0.5 * (e2[i, j, i, j] - e2[i, j, j, i])
    return e


def orbital_energies(e1, e2, occ_a):
    n = e1.shape[0]
    out = np.zeros(n)
    for i in range(n):
        acc = e1[i, i]
        for j in range(occ_a):
            acc += 2.0 * e2[i, j, i, j] - e2[i, j, j, i]
        out[i] = acc
    return out


@dataclass
class Dims:
    """Active dimensions; ``oa``/``ob`` occupied and ``va``/``vb`` virtual per spin."""
    froz: int
    occ_a: int
    occ_b: int
    orbs: int

    @property
    def oa(self):
        return self.occ_a - self.froz

    @property
    def ob(self):
        return self.occ_b - self.froz

    @property
    def va(self):
        return self.orbs - self.occ_a

    @property
    def vb(self):
        return self.orbs - self.occ_b

    @property
    def n(self):
        return self.orbs - self.froz


# Block shapes in the memory order of the Fortran arrays (read in C order).
BLOCK_SHAPES = {
    'T1A': ('oa', 'va'),
    'T1B': ('ob', 'vb'),
    'T2A': ('oa', 'oa', 'va', 'va'),
    'T2B': ('oa', 'ob', 'va', 'vb'),
    'T2C': ('ob', 'ob', 'vb', 'vb'),
    'T3A': ('oa', 'oa', 'oa', 'va', 'va', 'va'),
    'T3B': ('oa', 'oa', 'ob', 'va', 'va', 'vb'),
    'T3C': ('oa', 'ob', 'ob', 'va', 'vb', 'vb'),
    'T3D': ('ob', 'ob', 'ob', 'vb', 'vb', 'vb'),
    'T4A': ('oa',) * 4 + ('va',) * 4,
    'T4B': ('oa', 'oa', 'oa', 'ob', 'va', 'va', 'va', 'vb'),
    'T4C': ('oa', 'oa', 'ob', 'ob', 'va', 'va', 'vb', 'vb'),
    'T4D': ('oa', 'ob', 'ob', 'ob', 'va', 'vb', 'vb', 'vb'),
    'T4E': ('ob',) * 4 + ('vb',) * 4,
}

T_VEC_ORDER = ['T1A', 'T1B', 'T2A', 'T2B', 'T2C', 'T3A', 'T3B', 'T3C', 'T3D']
T4_ORDER = ['T4A', 'T4B', 'T4C', 'T4D', 'T4E']


class TLayout:
    """Offsets of the T blocks inside ``t_vec`` (``get_t_sizes``).

    ``t_size`` always includes the T3 blocks, also for CCSD, exactly as the
    reference allocates it.  T4 blocks (CCSDTQ) are kept outside ``t_vec``,
    like the reference's T4 scratch files, and are never part of DIIS.
    """

    def __init__(self, dims: Dims):
        self.dims = dims
        self.shape = {}
        self.offset = {}
        off = 0
        for b in T_VEC_ORDER:
            shp = tuple(getattr(dims, s) for s in BLOCK_SHAPES[b])
            self.shape[b] = shp
            self.offset[b] = off
            off += int(np.prod(shp))
        self.t_size = off
        # pos(1..10) as 1-based Fortran offsets
        self.pos = [self.offset[b] + 1 for b in T_VEC_ORDER] + [off + 1]
        self.t4_shape = {b: tuple(getattr(dims, s) for s in BLOCK_SHAPES[b]) for b in T4_ORDER}

    def size(self, b):
        return int(np.prod(self.shape[b])) if b in self.shape else int(np.prod(self.t4_shape[b]))

    def view(self, tvec, b):
        o = self.offset[b]
        return tvec[o:o + self.size(b)].reshape(self.shape[b])

    def vec_size(self, calc_type):
        """DIIS vector length (``solve_cc.f90:66-77``): T1+T2 for CCSD, else all."""
        if calc_type == 'CCSD':
            return self.offset['T3A']
        return self.t_size
