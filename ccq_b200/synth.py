"""Seeded synthetic closed-shell Hamiltonians in ccq's integral format.

Stand-in for real molecular integrals (none travel with this repository).
Draw order from ``numpy.random.default_rng(seed)``:
  1. B (L x N x N), symmetric: upper triangle incl. diagonal ~ N(0, sigma^2),
     mirrored;
  2. occupied orbital energies ~ U[-1.5, -0.5] (sorted ascending);
  3. virtual orbital energies ~ U[0.2, 2.0] (sorted ascending).
(pq|rs) = sum_L B^L_pq B^L_rs (positive semidefinite, 8-fold symmetric) and
h_pq = delta_pq eps_p - sum_{i occ} [2 (pq|ii) - (pi|iq)], so the closed-shell
Fock matrix is diag(eps).  E_nuc = 0.  ``lam`` scales the off-diagonal
B^L_pq by sqrt(lam) (bond-stretch family of the warm-start study).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import integrals as I


@dataclass
class SynthSpec:
    norb: int
    nel: int
    L: int
    sigma: float
    seed: int
    lam: float = 1.0

    @property
    def nvir(self):
        return 2 * self.norb - self.nel


# Workloads of the benchmark study (spatial orbitals, electrons, L, sigma, seed).
C0 = SynthSpec(20, 10, 40, 0.03, 0)      # CCSD, CPU-runnable size
C1 = SynthSpec(32, 14, 64, 0.03, 1)      # CCSD + CR-CC(2,3) size
C2 = SynthSpec(40, 16, 80, 0.025, 2)     # CCSDT, 40 spatial orbitals


def generate(spec: SynthSpec):
    """Returns (e1int[N,N], e2int[N,N,N,N] with e2int[i,j,a,b] = <ij|ab>, en_repul)."""
    rng = np.random.default_rng(spec.seed)
    N, L = spec.norb, spec.L
    B = np.zeros((L, N, N))
    iu = np.triu_indices(N)
    vals = rng.normal(0.0, spec.sigma, size=(L, len(iu[0])))
    B[:, iu[0], iu[1]] = vals
    B[:, iu[1], iu[0]] = vals
    if spec.lam != 1.0:
        off = ~np.eye(N, dtype=bool)
        B[:, off] *= np.sqrt(spec.lam)
    nocc = spec.nel // 2
    eps_o = np.sort(rng.uniform(-1.5, -0.5, size=nocc))
    eps_v = np.sort(rng.uniform(0.2, 2.0, size=N - nocc))
    eps = np.concatenate([eps_o, eps_v])
    chem = np.einsum('Lpq,Lrs->pqrs', B, B, optimize=True)
    occ = np.arange(nocc)
    J = np.einsum('pqii->pq', chem[:, :, occ][:, :, :, occ])
    K = np.einsum('piiq->pq', chem[:, occ][:, :, occ])
    h = np.diag(eps) - (2.0 * J - K)
    e2 = np.ascontiguousarray(chem.transpose(0, 2, 1, 3))   # <ij|ab> = (ia|jb)
    return h, e2, 0.0


def system(spec: SynthSpec, froz=0):
    """Spin blocks and Fock matrices ready for a solver (active range from froz)."""
    h, e2, enuc = generate(spec)
    occ = spec.nel // 2
    fa, fb = I.fock(h, e2, occ, occ)
    vaa, vab, vbb = I.spin_blocks(e2, froz)
    dims = I.Dims(froz, occ, occ, spec.norb)
    eref = I.hf_energy(h, e2, occ, occ) + enuc
    return dict(dims=dims, f_a=fa, f_b=fb, v_aa=vaa, v_ab=vab, v_bb=vbb, e_ref=eref, h=h, e2=e2)


def write_inputs(spec: SynthSpec, directory, calc_type, tol=1e-8, diis_space=5, max_iter=200, extra=()):
    import os
    h, e2, enuc = generate(spec)
    os.makedirs(directory, exist_ok=True)
    I.write_onebody(os.path.join(directory, 'onebody.inp'), h)
    I.write_twobody(os.path.join(directory, 'twobody.inp'), e2, enuc)
    with open(os.path.join(directory, f'{calc_type}.inp'), 'w') as fh:
        fh.write(f'froz=0\nnel={spec.nel}\nnvir={spec.nvir}\n')
        fh.write(f'onebody={directory}/onebody.inp\ntwobody={directory}/twobody.inp\n')
        fh.write(f'tol={tol}\ndiis_space={diis_space}\nmax_iterations={max_iter}\ncalc_type={calc_type}\n')
        for line in extra:
            fh.write(line + '\n')
    return os.path.join(directory, f'{calc_type}.inp')
