"""Shared builders for the tests (random and synthetic systems)."""
import numpy as np

from ccq_b200 import integrals as I


def random_system(n, occ_a, occ_b, seed, sigma=0.1, froz=0):
    rng = np.random.default_rng(seed)
    L = 2 * n
    B = rng.normal(0, sigma, (L, n, n))
    B = 0.5 * (B + B.transpose(0, 2, 1))
    chem = np.einsum('Lpq,Lrs->pqrs', B, B)
    e2 = chem.transpose(0, 2, 1, 3).copy()
    h = rng.normal(0, 0.05, (n, n))
    h = 0.5 * (h + h.T) + np.diag(np.linspace(-2.0, 1.0, n))
    fa, fb = I.fock(h, e2, occ_a, occ_b)
    vaa, vab, vbb = I.spin_blocks(e2, froz)
    return dict(h=h, e2=e2, f_a=fa, f_b=fb, v_aa=vaa, v_ab=vab, v_bb=vbb,
                dims=I.Dims(froz, occ_a, occ_b, n))


def random_t(dims, seed, scale=0.02, nmax=3):
    """Random amplitudes with the reference's antisymmetry (canonical + fill)."""
    from oracle import solver as S
    rng = np.random.default_rng(seed)
    lay = I.TLayout(dims)
    t = np.zeros(lay.t_size)
    for b in I.T_VEC_ORDER:
        if int(b[1]) > nmax:
            continue
        v = lay.view(t, b)
        v[...] = S.antisym_fill(b, rng.normal(0, scale, v.shape))
    t4 = {}
    if nmax >= 4:
        for b, shp in lay.t4_shape.items():
            t4[b] = S.antisym_fill(b, rng.normal(0, scale, shp))
    return t, t4


def fci_cluster_amplitudes(so, nmax=4):
    """Exact cluster amplitudes of the FCI ground state of a SpinOrbitalSystem.

    The FCI vector psi (Sz of the reference, <Phi|psi> = 1) gives C_n, its
    n-fold excitation coefficients in the amplitude convention of
    oracle.detcc; exp(T)|Phi> = psi then fixes T_n = C_n - [exp(T_1 + .. +
    T_{n-1})|Phi>]_n level by level.  Returns ({n: T_n[a.., i..]}, E_FCI - E_ref).
    """
    from oracle.detcc import DetCC
    dc = DetCC(so.h, so.v, so.O)
    psi, e = fci_state(so, dc)
    ts = {}
    for n in range(1, nmax + 1):
        C = dc.residual({}, n, w=psi)
        if ts:
            C = C - dc.residual({}, n, w=dc.exp_t(ts, dc.phi))
        ts[n] = C
    return ts, e


def fci_state(so, dc=None):
    """FCI ground state of a SpinOrbitalSystem in the Sz sector of the reference, as a Fock-space
    vector of oracle.detcc with <Phi|psi> = 1, and E_FCI - E_ref."""
    from oracle.detcc import DetCC
    dc = dc or DetCC(so.h, so.v, so.O)
    fs = dc.fs
    states = fs.states
    pc = np.array([bin(int(x)).count('1') for x in states])
    sel = np.where(pc == so.O)[0]
    # Sz sector of the reference: as many alpha spin orbitals occupied as in the reference
    amask = sum(1 << p for p in range(so.N) if so.spin[p] == 0)
    nref = bin(((1 << so.O) - 1) & amask).count('1')
    sel = sel[np.array([bin(int(x) & amask).count('1') for x in states[sel]]) == nref]
    H = np.zeros((len(sel), len(sel)))
    for k, x in enumerate(sel):
        e = np.zeros(1 << so.N)
        e[x] = 1.0
        H[:, k] = dc.apply_h(e)[sel]
    w, U = np.linalg.eigh(0.5 * (H + H.T))
    psi = np.zeros(1 << so.N)
    psi[sel] = U[:, 0]
    psi /= psi[(1 << so.O) - 1]
    return psi, float(w[0]) - dc.e_ref()
