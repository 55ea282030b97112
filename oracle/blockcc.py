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
        self.sizes = {'oa': dims.oa, 'ob': dims.ob, 'va': dims.va, 'vb': dims.vb, 'n': dims.n, '1': 1, '0': 0}
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
        self.buf['ONES'][...] = 1.0
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

    def update(self, tvec):
        # everything except the energy phase
        ops = self.plan['ops']
        k = [i for i, o in enumerate(ops) if o[0] == 'PHASE' and o[1] == 'energy'][0]
        self.run(tvec, ops[:k])

    def energy(self, tvec):
        ops = self.plan['ops']
        k = [i for i, o in enumerate(ops) if o[0] == 'PHASE' and o[1] == 'energy'][0]
        self.run(tvec, ops[k:])
        return float(self.buf['E'])

    def solve(self, diis_space=5, max_iter=60, tol=1e-8, log=None):
        tvec = np.zeros(self.layout.t_size)
        vs = self.layout.vec_size(self.method)
        e, it, failed, hist = S.jacobi_iter(self.update, self.energy, tvec, vs, diis_space, max_iter, tol, log)
        return e, it, failed, hist, tvec
