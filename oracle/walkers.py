"""FCIQMC walker files and their cluster analysis on the CPU (test infrastructure only).

* ``write``  a Fock-space state of ``oracle.detcc`` (bit P = spin orbital P of
             a ``SpinOrbitalSystem``: alpha occupied, beta occupied, alpha
             virtual, beta virtual) as the records ``c_id coef occ_1 .. occ_m``
             that ``parse_fciqmc_c3`` reads (``src/ext_cor/ext_cor.f90:205-208``):
             spin orbitals numbered from the first unfrozen one, odd alpha and
             even beta, each determinant's creators in ascending order of that
             numbering, so its coefficient takes the parity of the reordering.
* ``read``   the file back into the Fock space (the inverse reordering), and
             the cluster amplitudes of the state: C_n, its n-fold excitation
             coefficients over the Hartree-Fock one, and T_n = C_n -
             [exp(T_1 + .. + T_{n-1})|Phi>]_n rank by rank (the relation
             ``cluster_analysis_up_t3``, ``src/ext_cor/cluster_analysis.f90:10-258``,
             and ``drive_t4_contraction``, ``src/ext_cor/contract_t4.f90:241-479``,
             evaluate), returned as spin blocks.

This route shares nothing with the native reader: it never computes the
reference's ``excitation_sign_qmc`` parity and applies exp(T) in Fock space
instead of a cluster formula.  Like the reference, repeated determinants keep
their last coefficient up to triples and add up for quadruples.  Only
``tests/`` use this module.
"""
from __future__ import annotations

import numpy as np

from ccq_b200 import integrals as I


def _parity(seq):
    inv = 0
    for a in range(len(seq)):
        for b in range(a + 1, len(seq)):
            inv += seq[a] > seq[b]
    return inv & 1


def _file_number(so, P):
    k, s = so.sp[P]
    return 2 * (k + 1) - 1 if s == 0 else 2 * (k + 1)


def write(path, so, psi, tol=None, extra=()):
    """Records for every basis state with psi != 0 (or |psi| > tol); ``extra`` lines are appended."""
    lines = []
    cid = 0
    for x in np.nonzero(psi)[0]:
        c = float(psi[x])
        if tol is not None and abs(c) <= tol:
            continue
        pos = [P for P in range(so.N) if (int(x) >> P) & 1]
        nums = [_file_number(so, P) for P in pos]
        sign = -1.0 if _parity(nums) else 1.0
        cid += 1
        lines.append(f'{cid} {sign * c: .17e} ' + ' '.join(str(v) for v in sorted(nums)))
    lines += list(extra)
    with open(path, 'w') as fh:
        fh.write('\n'.join(lines) + '\n')


def read(path, so, nel_active):
    """Fock-space vector of a walker file (records as the reference reads them) and the level of each state."""
    inv = {_file_number(so, P): P for P in range(so.N)}
    ref = (1 << so.O) - 1
    psi = np.zeros(1 << so.N)
    with open(path) as fh:
        toks = fh.read().split('\n')
    k = 0
    m = nel_active
    while True:
        acc = []
        while len(acc) < m + 2 and k < len(toks):
            acc += toks[k].replace(',', ' ').split()
            k += 1
        if len(acc) < m + 2:
            break
        try:
            int(acc[0])
            coef = float(acc[1].replace('D', 'E').replace('d', 'e'))
            nums = [int(t) for t in acc[2:m + 2]]
        except ValueError:
            break
        pos = [inv[v] for v in sorted(nums)]
        x = sum(1 << P for P in pos)
        c = -coef if _parity(pos) else coef
        level = bin(x ^ ref).count('1') // 2
        if level == 4:
            psi[x] += c
        else:
            psi[x] = c
    return psi


def cluster_blocks(so, psi, nmax=4):
    """{block name: T block} of the state psi (T1..T3 in t_vec blocks, T4A..T4E)."""
    from oracle.detcc import DetCC
    ref = (1 << so.O) - 1
    if psi[ref] == 0.0:
        raise ValueError('the Hartree-Fock coefficient is not in the file')
    dc = DetCC(so.h, so.v, so.O)
    w = psi / psi[ref]
    ts = {}
    for n in range(1, nmax + 1):
        C = dc.residual({}, n, w=w)
        if ts:
            C = C - dc.residual({}, n, w=dc.exp_t(ts, dc.phi))
        ts[n] = C
    names = I.T_VEC_ORDER + (I.T4_ORDER if nmax >= 4 else [])
    names = [b for b in names if int(b[1]) <= nmax]
    return so.to_blocks(ts, names)
