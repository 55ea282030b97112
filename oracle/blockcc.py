"""Spin-blocked numpy executor of the contraction plan (test infrastructure).

Interprets the same plan text that ``libccq_b200`` runs on the GPU, with
``numpy.einsum`` for every GETT, on the reference's data layout (full-range
antisymmetrised integral blocks, T blocks in ``t_vec`` order).  It is the
CPU restatement used at sizes the dense spin-orbital oracle cannot reach, and
the timed CPU baseline of ``bench.py``.  Its agreement with
``oracle/densecc.py`` (no spin integration) on small systems is what pins the
plan compiler.  Only ``tests/`` and ``bench.py``'s CPU leg use this module.
"""
from __future__ import annotations

import itertools

import numpy as np

from ccq_b200 import integrals as I
from oracle import solver as S

LETTERS = 'abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ'


def parse_view(tok):
    name, rest = tok.split('[', 1)
    rest = rest.rstrip(']')
    axes = []
    if rest:
        for a in rest.split(','):
            start = '0'
            if '@' in a:
                a, start = a.split('@')
            lab, size = a.split(':')
            axes.append((lab, size, start))
    return name, axes


def parse_plan(text):
    lines = text.strip().split('\n')
    head = lines[0].split()
    plan = {'method': head[1], 'buffers': {}, 'ops': []}
    k = 1
    while lines[k].startswith('BUF'):
        p = lines[k].split()
        nd = int(p[3])
        plan['buffers'][p[1]] = (p[2], p[4:4 + nd])   # a trailing G= (antisymmetric axes) is a GPU hint
        k += 1
    assert lines[k].startswith('OPS')
    k += 1
    while lines[k] != 'END':
        p = lines[k].split()
        if p[0] == 'GETT':
            # a trailing R= token restricts index tuples on the GPU; the full sum is identical
            tag = p[6] if len(p) > 6 and not p[6].startswith('R=') else ''
            plan['ops'].append(('GETT', float(p[1]), int(p[2]), parse_view(p[3]), parse_view(p[4]), parse_view(p[5]), tag))
            k += 1
        elif p[0] == 'ASSEMBLE':
            nt = int(p[3])
            terms = []
            for j in range(nt):
                q = lines[k + 1 + j].split()
                terms.append((float(q[1]), parse_view(q[2])))
            plan['ops'].append(('ASSEMBLE', p[1], p[2], terms))
            k += 1 + nt
        else:
            plan['ops'].append(tuple(p))
            k += 1
    return plan


def check_written_before_read(plan):
    """Every work buffer (Z*, X*) must be overwritten (beta=0) before it is read."""
    written = set()
    for op in plan['ops']:
        if op[0] == 'GETT':
            _, alpha, beta, cv, av, bv, tag = op
            for v in (av, bv):
                if v[0][0] in 'ZX' and v[0] not in written:
                    raise ValueError(f'{v[0]} read before written')
            if cv[0][0] in 'ZX':
                if beta and cv[0] not in written:
                    raise ValueError(f'{cv[0]} accumulated before written')
                written.add(cv[0])
        elif op[0] == 'ASSEMBLE':
            for _, v in op[3]:
                if v[0][0] in 'ZX' and v[0] not in written:
                    raise ValueError(f'{v[0]} read by assemble before written')
        elif op[0] == 'PHASE':
            written = set()


class BlockCC:
    """Runs the plan with numpy on one system."""

    def __init__(self, plan_text, f_a, f_b, v_aa, v_ab, v_bb, dims: I.Dims, method, shift=0.0, count_flops=False):
        self.plan = parse_plan(plan_text)
        self.dims = dims
        self.method = method
        self.shift = shift
        self.layout = I.TLayout(dims)
        fr = dims.froz
        self.sizes = {'oa': dims.oa, 'ob': dims.ob, 'va': dims.va, 'vb': dims.vb, 'n': dims.n, '1': 1, '0': 0, '4': 4}
        self.buf = {}
        for name, (kind, dd) in self.plan['buffers'].items():
            shape = tuple(self.sizes[d] for d in dd)
            if kind == 'amp' and name in self.layout.shape:
                continue   # views into t_vec
            self.buf[name] = np.zeros(shape)
        fa = f_a[fr:, fr:]
        fb = f_b[fr:, fr:]
        oa, ob = dims.oa, dims.ob
        self.buf['FA0'][...] = fa
        self.buf['FB0'][...] = fb
        self.buf['VAA0'][...] = v_aa
        self.buf['VAB0'][...] = v_ab
        self.buf['VBB0'][...] = v_bb
        self.buf['HA0'][...] = fa - np.einsum('piqi->pq', v_aa[:, :oa, :, :oa]) - np.einsum('piqi->pq', v_ab[:, :ob, :, :ob])
        self.buf['HB0'][...] = fb - np.einsum('piqi->pq', v_bb[:, :ob, :, :ob]) - np.einsum('ipiq->pq', v_ab[:oa, :, :oa, :])
        for name, (kind, dd) in self.plan['buffers'].items():
            if kind == 'ones':
                self.buf[name][...] = 1.0
        self.fdiag_a = np.diag(fa).copy()
        self.fdiag_b = np.diag(fb).copy()
        self.flops = 0
        self.count_flops = count_flops
        check_written_before_read(self.plan)

    def _array(self, name, tvec):
        if name in self.layout.shape:
            return self.layout.view(tvec, name)
        return self.buf[name]

    def _view(self, v, tvec):
        name, axes = v
        arr = self._array(name, tvec)
        sl = []
        for lab, size, start in axes:
            s0 = self.sizes[start]
            sl.append(slice(s0, s0 + self.sizes[size]))
        return (arr[tuple(sl)] if sl else arr[...]), [a[0] for a in axes]

    def run(self, tvec, ops=None):
        for op in (ops or self.plan['ops']):
            self._op(op, tvec)

    def _op(self, op, tvec):
        kind = op[0]
        if kind == 'GETT':
            _, alpha, beta, cv, av, bv, tag = op
            C, cl = self._view(cv, tvec)
            A, al = self._view(av, tvec)
            B, bl = self._view(bv, tvec)
            letters = {}
            for l in al + bl + cl:
                if l not in letters:
                    letters[l] = LETTERS[len(letters)]
            sub = ''.join(letters[l] for l in al) + ',' + ''.join(letters[l] for l in bl) + '->' + ''.join(letters[l] for l in cl)
            r = alpha * np.einsum(sub, A, B, optimize=True)
            if self.count_flops:
                sz = {}
                for arr, ls in ((A, al), (B, bl)):
                    for d, l in zip(arr.shape, ls):
                        sz[l] = d
                f = 2
                for l in sz:
                    f *= sz[l]
                self.flops += f
            if beta:
                C += r
            else:
                C[...] = r
        elif kind == 'ASSEMBLE':
            _, block, mode, terms = op
            T = self._array(block, tvec)
            level = int(block[1])
            target = [f'i{k}' for k in range(level)] + [f'a{k}' for k in range(level)]
            R = np.zeros(T.shape)
            for coef, v in terms:
                X, xl = self._view(v, tvec)
                R += coef * np.einsum(''.join(LETTERS[target.index(l)] for l in xl) + '->' + LETTERS[:2 * level], X)
            if mode == 'jacobi':
                D = S.denominator(block, T.shape, self.fdiag_a, self.fdiag_b, self.dims, self.shift)
                T[...] = S.jacobi_block(block, T, R, D)
            else:
                T[...] = S.antisym_fill(block, np.where(S.canonical_mask(block, R.shape), R, 0.0))
        elif kind == 'COPY':
            self.buf[op[1]][...] = self.buf[op[2]]
        elif kind == 'ZERO':
            self._array(op[1], tvec)[...] = 0.0
        elif kind == 'PHASE':
            pass
        else:
            raise ValueError(kind)

    def phase_index(self, name):
        ops = self.plan['ops']
        hits = [i for i, o in enumerate(ops) if o[0] == 'PHASE' and o[1] == name]
        return hits[0] if hits else len(ops)

    def update(self, tvec):
        # everything before the energy phase
        self.run(tvec, self.plan['ops'][:self.phase_index('energy')])

    def energy(self, tvec):
        # the energy phase (a CR-CC(2,3) plan continues after its 'crcc' marker)
        self.run(tvec, self.plan['ops'][self.phase_index('energy'):self.phase_index('crcc')])
        return float(self.buf['E'])

    def solve(self, diis_space=5, max_iter=60, tol=1e-8, log=None):
        tvec = np.zeros(self.layout.t_size)
        vs = self.layout.vec_size(self.method)
        e, it, failed, hist = S.jacobi_iter(self.update, self.energy, tvec, vs, diis_space, max_iter, tol, log)
        return e, it, failed, hist, tvec


L_BLOCKS = ('L1A', 'L1B', 'L2A', 'L2B', 'L2C')


class BlockCRCC(BlockCC):
    """Runs a CR-CC(2,3) plan (``PlanBuilder.build_crcc``) with numpy.

    The CC sweep and energy are those of ``BlockCC``; the ops after the
    ``crcc`` marker are: the ``ljacobi`` assemble (left Jacobi step with the
    Hbar one-body diagonal, ``shift - E_cor`` and the sum of LH^2 of every
    stored element into LN), ``CRDIAG`` (the Hbar diagonals and ``cal_d3``
    sums of ``src/mm_correct.f90:346-481`` in spin-blocked form), ``LENERGY``
    and ``CRCC`` (the four-denominator sums of ``crcc23``,
    ``src/mm_correct.f90:110-338``).  Lambda lives in ``lvec`` with the T1/T2
    layout of ``t_vec``.
    """

    def __init__(self, plan_text, f_a, f_b, v_aa, v_ab, v_bb, dims: I.Dims, shift=0.0, active=None):
        super().__init__(plan_text, f_a, f_b, v_aa, v_ab, v_bb, dims, 'CCSD', shift)
        # CC(t;3): (act_occ_b, act_unocc_a); the sums leave out the triples of that active space
        self.active = active
        self.lvec = np.zeros(self.layout.t_size)
        for b in L_BLOCKS:
            self.buf[b] = self.layout.view(self.lvec, 'T' + b[1:])

    # -- the CR-CC(2,3) operations ----------------------------------------------
    def _op(self, op, tvec):
        kind = op[0]
        if kind == 'ASSEMBLE' and op[2] == 'ljacobi':
            _, block, mode, terms = op
            T = self._array(block, tvec)
            level = int(block[1])
            target = [f'i{k}' for k in range(level)] + [f'a{k}' for k in range(level)]
            R = np.zeros(T.shape)
            for coef, v in terms:
                X, xl = self._view(v, tvec)
                R += coef * np.einsum(''.join(LETTERS[target.index(l)] for l in xl) + '->' + LETTERS[:2 * level], X)
            name = 'T' + block[1:]
            R = S.antisym_fill(name, np.where(S.canonical_mask(name, R.shape), R, 0.0))
            self.buf['LN'][...] += np.sum(R * R)
            D = S.denominator(name, T.shape, self.buf['HDA'], self.buf['HDB'], self.dims,
                              self.shift - float(self.buf['ECOR']))
            T[...] = S.jacobi_block(name, T.copy(), R, D)
        elif kind == 'CRDIAG':
            self._crdiag(tvec)
        elif kind == 'LENERGY':
            self.buf['EL'][...] = np.sqrt(float(self.buf['LN'])) + float(self.buf['ECOR'])
        elif kind == 'CRCC':
            self._crcc(op[1])
        else:
            super()._op(op, tvec)

    def _crdiag(self, tvec):
        b = self.buf
        oa, ob, n = self.dims.oa, self.dims.ob, self.dims.n
        t2a = self.layout.view(tvec, 'T2A')
        t2b = self.layout.view(tvec, 'T2B')
        t2c = self.layout.view(tvec, 'T2C')
        vaa = b['VAA0'][:oa, :oa, oa:, oa:]
        vab = b['VAB0'][:oa, :ob, oa:, ob:]
        vbb = b['VBB0'][:ob, :ob, ob:, ob:]
        es = np.einsum
        fa, fb = np.diag(b['FA']), np.diag(b['FB'])
        b['HDA'][:oa] = fa[:oa] + 0.5 * es('imef,imef->i', vaa, t2a) + es('imef,imef->i', vab, t2b)
        b['HDA'][oa:] = fa[oa:] - 0.5 * es('mnaf,mnaf->a', vaa, t2a) - es('mnaf,mnaf->a', vab, t2b)
        b['HDB'][:ob] = fb[:ob] + 0.5 * es('imef,imef->i', vbb, t2c) + es('mief,mief->i', vab, t2b)
        b['HDB'][ob:] = fb[ob:] - 0.5 * es('mnaf,mnaf->a', vbb, t2c) - es('mnfa,mnfa->a', vab, t2b)
        VA, VB, VM = b['VAA'], b['VBB'], b['VAB']
        h = b['H2AA']
        h[:oa, :oa] = es('ijij->ij', VA[:oa, :oa, :oa, :oa]) + 0.5 * es('ijef,ijef->ij', vaa, t2a)
        h[oa:, oa:] = es('abab->ab', VA[oa:, oa:, oa:, oa:]) + 0.5 * es('mnab,mnab->ab', vaa, t2a)
        h[oa:, :oa] = (es('aiai->ai', VA[oa:, :oa, oa:, :oa]) - es('inaf,inaf->ai', vaa, t2a)
                       - es('inaf,inaf->ai', vab, t2b))
        h[:oa, oa:] = h[oa:, :oa].T
        h = b['H2BB']
        h[:ob, :ob] = es('ijij->ij', VB[:ob, :ob, :ob, :ob]) + 0.5 * es('ijef,ijef->ij', vbb, t2c)
        h[ob:, ob:] = es('abab->ab', VB[ob:, ob:, ob:, ob:]) + 0.5 * es('mnab,mnab->ab', vbb, t2c)
        h[ob:, :ob] = (es('aiai->ai', VB[ob:, :ob, ob:, :ob]) - es('inaf,inaf->ai', vbb, t2c)
                       - es('nifa,nifa->ai', vab, t2b))
        h[:ob, ob:] = h[ob:, :ob].T
        h = b['H2AB']
        h[:oa, :ob] = es('ijij->ij', VM[:oa, :ob, :oa, :ob]) + es('ijef,ijef->ij', vab, t2b)
        h[oa:, ob:] = es('abab->ab', VM[oa:, ob:, oa:, ob:]) + es('mnab,mnab->ab', vab, t2b)
        h[oa:, :ob] = es('aiai->ai', VM[oa:, :ob, oa:, :ob]) - es('niaf,niaf->ai', vab, t2b)
        h[:oa, ob:] = es('iaia->ia', VM[:oa, ob:, :oa, ob:]) - es('infa,infa->ia', vab, t2b)
        b['W1A'][oa:, :oa, :oa] = es('pqxe,pqxe->xpq', vaa, t2a)
        b['W1B'][oa:, :oa, :ob] = es('pqxe,pqxe->xpq', vab, t2b)
        b['W1C'][ob:, :oa, :ob] = es('pqex,pqex->xpq', vab, t2b)
        e0 = max(0, oa + 1 - ob)   # cal_d3's d3d1 loop starts at orbital occ_a + 2
        b['W1D'][ob:, :ob, :ob] = es('pqxe,pqxe->xpq', vbb[:, :, :, e0:], t2c[:, :, :, e0:])
        b['W2A'][oa:, oa:, :oa] = es('ymxz,ymxz->xzy', vaa, t2a)
        b['W2B'][oa:, ob:, :oa] = es('ymxz,ymxz->xzy', vab, t2b)
        b['W2C'][oa:, ob:, :ob] = es('myxz,myxz->xzy', vab, t2b)
        b['W2D'][ob:, ob:, :ob] = es('ymxz,ymxz->xzy', vbb, t2c)

    def _crcc(self, x):
        b = self.buf
        name = 'T3' + x
        M, L = b['M3' + x], b['L3' + x]
        spins = S.block_spins(name)
        off = [self.dims.oa, self.dims.ob]
        keep = S.canonical_mask(name, M.shape)
        if self.active is not None:
            # crcc23's skip of the active-space triples (src/mm_correct.f90:131,190,244,300)
            from oracle.densecc import active_mask
            keep = keep & ~active_mask(name, M.shape, self.dims, self.active)
        idx = np.nonzero(keep)
        lm = L[idx] * M[idx]
        occ = [idx[k] for k in range(3)]
        vir = [idx[3 + k] + off[spins[k]] for k in range(3)]
        fdg = [self.fdiag_a, self.fdiag_b]
        hd = [b['HDA'], b['HDB']]

        def h2(s1, p, s2, q):
            if s1 == 0 and s2 == 0:
                return b['H2AA'][p, q]
            if s1 == 1 and s2 == 1:
                return b['H2BB'][p, q]
            return b['H2AB'][p, q] if s1 == 0 else b['H2AB'][q, p]
        w1 = {(0, 0, 0): 'W1A', (0, 0, 1): 'W1B', (1, 0, 1): 'W1C', (1, 1, 1): 'W1D'}
        w2 = {(0, 0, 0): 'W2A', (0, 1, 0): 'W2B', (0, 1, 1): 'W2C', (1, 1, 1): 'W2D'}
        da = sum(fdg[spins[k]][occ[k]] - fdg[spins[k]][vir[k]] for k in range(3))
        db = sum(hd[spins[k]][occ[k]] - hd[spins[k]][vir[k]] for k in range(3))
        dc = db.copy()
        for k, l in itertools.combinations(range(3), 2):
            dc -= h2(spins[k], occ[k], spins[l], occ[l]) + h2(spins[k], vir[k], spins[l], vir[l])
        for k in range(3):
            for l in range(3):
                dc += h2(spins[k], vir[k], spins[l], occ[l])
        dd = dc.copy()
        for k in range(3):
            for p, q in itertools.combinations(range(3), 2):
                key = (spins[k], spins[p], spins[q])
                if key in w1:
                    dd += b[w1[key]][vir[k], occ[p], occ[q]]
        for p, q in itertools.combinations(range(3), 2):
            for k in range(3):
                key = (spins[p], spins[q], spins[k])
                if key in w2:
                    dd += b[w2[key]][vir[p], vir[q], occ[k]]
        for q, d in enumerate((da, db, dc, dd)):
            b['E23'][q] += float(np.sum(lm / d))

    # -- drivers ---------------------------------------------------------------------
    def lambda_init(self, tvec, e_cor):
        ops = self.plan['ops']
        self.buf['ECOR'][...] = e_cor
        self.buf['E23'][...] = 0.0
        self.lvec[...] = 0.0
        self.run(tvec, ops[self.phase_index('crcc'):self.phase_index('lambda')])

    def lambda_update(self, lvec, tvec):
        ops = self.plan['ops']
        assert lvec is self.lvec
        self.run(tvec, ops[self.phase_index('lambda'):self.phase_index('lenergy')])

    def lambda_energy(self, lvec, tvec):
        ops = self.plan['ops']
        self.run(tvec, ops[self.phase_index('lenergy'):self.phase_index('triplesA')])
        return float(self.buf['EL'])

    def crcc23(self, tvec):
        ops = self.plan['ops']
        self.buf['E23'][...] = 0.0
        self.run(tvec, ops[self.phase_index('triplesA'):])
        return self.buf['E23'].copy()

    def solve_left(self, tvec, e_cor, diis_space=5, max_iter=60, tol=1e-8):
        self.lambda_init(tvec, e_cor)
        vs = self.layout.vec_size('CCSD')
        return S.jacobi_iter(lambda l: self.lambda_update(l, tvec), lambda l: self.lambda_energy(l, tvec),
                             self.lvec, vs, diis_space, max_iter, tol)
