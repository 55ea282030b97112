"""Plan compiler: spin-orbital residuals -> spin-blocked contraction plan.

The reference's generated update routines (``src/cc/t*_update.f90``) are,
per spin block, sequences of ``reorder_shift``/``reorder_stripe`` (permute a
slice), ``egemm`` (``dgemm('t','n')``), ``sum_stripe`` (permuted accumulate)
and a closing Jacobi step.  This compiler produces the same kind of sequence
as data: every diagram becomes one or more GETT operations (a GEMM whose
operands and result are strided, permuted views of resident tensors, so no
permute copies are made), every antisymmetriser becomes a list of permuted
views read by the block's closing ASSEMBLE (residual gather + Jacobi + fill).

Spin integration: each spin-orbital label gets a spin; external spins are
fixed by the target block, dummy spins are summed; every factor is mapped to
its stored spin block (v_aa, v_ab, v_bb, T2A, T2B, ...) with the index
permutation and sign of the canonical (alpha-first) ordering.

The plan is symbolic in the dimension tokens ``oa ob va vb n`` and is
serialised as text; ``libccq_b200`` instantiates it for concrete sizes.
"""
from __future__ import annotations

import itertools
import re
from dataclasses import dataclass, field
from fractions import Fraction

from . import wick

SIZE = {('o', 0): 'oa', ('o', 1): 'ob', ('v', 0): 'va', ('v', 1): 'vb'}
START = {('o', 0): '0', ('o', 1): '0', ('v', 0): 'oa', ('v', 1): 'ob'}


def _sp(label):
    return 'o' if label[0] in 'io' else 'v'


@dataclass
class Axis:
    label: str
    size: str
    start: str = '0'

    def text(self):
        s = f'{self.label}:{self.size}'
        if self.start != '0':
            s += f'@{self.start}'
        return s


@dataclass
class View:
    buf: str
    axes: list

    def text(self):
        return f"{self.buf}[{','.join(a.text() for a in self.axes)}]"

    def labels(self):
        return [a.label for a in self.axes]


@dataclass
class Gett:
    c: View
    a: View
    b: View
    alpha: float
    beta: int
    tag: str = ''
    restrict: list = field(default_factory=list)   # label groups enumerated in increasing order

    def text(self):
        r = ''
        if self.restrict:
            r = ' R=' + ';'.join(','.join(g) for g in self.restrict)
        return f'GETT {self.alpha!r} {self.beta} {self.c.text()} {self.a.text()} {self.b.text()} {self.tag}{r}'.rstrip()


@dataclass
class Assemble:
    block: str
    mode: str                 # 'jacobi' or 'copy'
    terms: list = field(default_factory=list)   # (coef, View with target labels)

    def text(self):
        out = [f'ASSEMBLE {self.block} {self.mode} {len(self.terms)}']
        for c, v in self.terms:
            out.append(f'TERM {float(c)!r} {v.text()}')
        return '\n'.join(out)


@dataclass
class Simple:
    kind: str
    args: tuple

    def text(self):
        return ' '.join([self.kind] + [str(a) for a in self.args])


BLOCK_DIMS = {
    'T1A': ('oa', 'va'), 'T1B': ('ob', 'vb'),
    'T2A': ('oa', 'oa', 'va', 'va'), 'T2B': ('oa', 'ob', 'va', 'vb'), 'T2C': ('ob', 'ob', 'vb', 'vb'),
    'T3A': ('oa', 'oa', 'oa', 'va', 'va', 'va'), 'T3B': ('oa', 'oa', 'ob', 'va', 'va', 'vb'),
    'T3C': ('oa', 'ob', 'ob', 'va', 'vb', 'vb'), 'T3D': ('ob', 'ob', 'ob', 'vb', 'vb', 'vb'),
    'T4A': ('oa',) * 4 + ('va',) * 4, 'T4B': ('oa', 'oa', 'oa', 'ob', 'va', 'va', 'va', 'vb'),
    'T4C': ('oa', 'oa', 'ob', 'ob', 'va', 'va', 'vb', 'vb'), 'T4D': ('oa', 'ob', 'ob', 'ob', 'va', 'vb', 'vb', 'vb'),
    'T4E': ('ob',) * 4 + ('vb',) * 4,
}
# left (lambda) amplitudes share the layout of T1/T2; the triples moments M3x and
# left projections L3x of CR-CC(2,3) that of T3x
for _b in ('1A', '1B', '2A', '2B', '2C'):
    BLOCK_DIMS['L' + _b] = BLOCK_DIMS['T' + _b]
for _b in ('A', 'B', 'C', 'D'):
    BLOCK_DIMS['M3' + _b] = BLOCK_DIMS['T3' + _b]
    BLOCK_DIMS['L3' + _b] = BLOCK_DIMS['T3' + _b]


def block_spins(name):
    n = int(name[1])
    nb = 'ABCDE'.index(name[2])
    return [0] * (n - nb) + [1] * nb


def _psign(p):
    s = 1
    p = list(p)
    for i in range(len(p)):
        for j in range(i + 1, len(p)):
            if p[j] < p[i]:
                s = -s
    return s


def _stable_spin_sort(labels, spin):
    order = sorted(range(len(labels)), key=lambda k: spin[labels[k]])
    return [labels[k] for k in order], _psign(order)


def map_factor(name, labels, spin, undressed=False):
    """Stored view of one spin-orbital factor for a spin assignment, or None.

    Returns (sign, View) with axes labelled by the term's labels.
    """
    def ax(l):
        key = (_sp(l), spin[l])
        return Axis(l, SIZE[key], START[key])

    if name == 'f':
        p, q = labels
        if spin[p] != spin[q]:
            return None
        buf = ('FA' if spin[p] == 0 else 'FB') + ('0' if undressed else '')
        return 1, View(buf, [ax(p), ax(q)])
    if name == 'v':
        p, q, r, s = labels
        sp = (spin[p], spin[q], spin[r], spin[s])
        z = '0' if undressed else ''
        if sp == (0, 0, 0, 0):
            return 1, View('VAA' + z, [ax(p), ax(q), ax(r), ax(s)])
        if sp == (1, 1, 1, 1):
            return 1, View('VBB' + z, [ax(p), ax(q), ax(r), ax(s)])
        if sp == (0, 1, 0, 1):
            return 1, View('VAB' + z, [ax(p), ax(q), ax(r), ax(s)])
        if sp == (1, 0, 1, 0):
            return 1, View('VAB' + z, [ax(q), ax(p), ax(s), ax(r)])
        if sp == (0, 1, 1, 0):
            return -1, View('VAB' + z, [ax(p), ax(q), ax(s), ax(r)])
        if sp == (1, 0, 0, 1):
            return -1, View('VAB' + z, [ax(q), ax(p), ax(r), ax(s)])
        return None
    # amplitudes: (vir..., occ...)
    n = len(labels) // 2
    vl = list(labels[:n])
    ol = list(labels[n:])
    if sorted(spin[l] for l in vl) != sorted(spin[l] for l in ol):
        return None
    vs, sv = _stable_spin_sort(vl, spin)
    os_, so = _stable_spin_sort(ol, spin)
    nb = sum(spin[l] for l in vl)
    block = name[0].upper() + f'{n}' + 'ABCDE'[nb]   # t<n> -> T blocks, l<n> -> L blocks
    axes = [Axis(l, SIZE[('o', spin[l])]) for l in os_] + [Axis(l, SIZE[('v', spin[l])]) for l in vs]
    return sv * so, View(block, axes)


def antisym_groups(view):
    """Label groups in which a stored view is antisymmetric (ordered by axis).

    T blocks: labels on one same-spin run of the occupied or virtual half.
    VAA/VBB (dressed or not): the bra pair (axes 0,1) and the ket pair (2,3)
    when both axes cover the same orbital range.  Intermediates: none.
    """
    labs = view.labels()
    if len(set(labs)) != len(labs):
        return []
    b = view.buf
    out = []
    if b[0] in 'TL' and len(b) == 3 and b[1].isdigit():
        n = int(b[1])
        spins = block_spins(b)
        for half in (0, n):
            start = 0
            for k in range(1, n + 1):
                if k == n or spins[k] != spins[start]:
                    if k - start >= 2:
                        out.append(tuple(labs[half + q] for q in range(start, k)))
                    start = k
    elif b in ('VAA', 'VBB', 'VAA0', 'VBB0'):
        for p, q in ((0, 1), (2, 3)):
            ap, aq = view.axes[p], view.axes[q]
            if ap.size == aq.size and ap.start == aq.start:
                out.append((labs[p], labs[q]))
    return out


def _refine(partitions, labels):
    """Common refinement of label groupings: labels stay together only if grouped in all."""
    key = {l: () for l in labels}
    for groups in partitions:
        gid = {}
        for k, g in enumerate(groups):
            for l in g:
                gid[l] = k
        for l in labels:
            key[l] = key[l] + (gid.get(l, ('solo', l)),)
    buckets = {}
    for l in labels:
        buckets.setdefault(key[l], []).append(l)
    return [tuple(v) for v in buckets.values() if len(v) >= 2]


SIZES_C2 = {'oa': 8, 'ob': 8, 'va': 32, 'vb': 32, 'n': 40, '1': 1}


def _numel(view, sizes):
    out = 1
    for a in view.axes:
        out *= sizes[a.size]
    return out


def _label_size(views, sizes):
    d = {}
    for v in views:
        for a in v.axes:
            d[a.label] = sizes[a.size]
    return d


class PlanBuilder:
    def __init__(self, method, rhf=False, est_sizes=None, workers=None):
        self.workers = workers
        self.method = method
        self.rhf = rhf
        self.tranks = wick.METHOD_TRANKS[method]
        self.nmax = max(self.tranks)
        self.sizes = est_sizes or SIZES_C2
        self.buffers = {}
        self.ops = []
        self.nz = 0
        self.nx = 0
        self.flops = 0
        self.zgroups = {}
        self.lam_last = False   # contract lambda factors last (their partners then form T-only intermediates)

    # -- buffers --------------------------------------------------------------
    def buf(self, name, kind, dims):
        self.buffers[name] = (kind, tuple(dims))
        return name

    def new_z(self, dims):
        name = f'Z{self.nz}'
        self.nz += 1
        return self.buf(name, 'work', dims)

    def new_x(self, dims):
        name = f'X{self.nx}'
        self.nx += 1
        return self.buf(name, 'work', dims)

    # -- spin-summed contraction chains --------------------------------------
    def _order(self, base):
        """Order of cluster factors minimising the spin-orbital GEMM cost."""
        so = {'o': 2 * self.sizes['oa'], 'v': 2 * self.sizes['va']}
        best = None
        for order in itertools.permutations(range(1, len(base))):
            if self.lam_last and any(base[k][0][0] == 'l' for k in order[:-1]):
                continue
            cur = set(base[0][1])
            cost = 0
            for k in order:
                tl = set(base[k][1])
                sh = cur & tl
                c = 1
                for l in cur | tl:
                    c *= so[_sp(l)]
                cost += c
                cur = (cur | tl) - sh
            if best is None or cost < best[0]:
                best = (cost, order)
        return best[1]

    def emit_chain(self, base, espin, dst, scale, tag, beta, undressed=False):
        """Emit GETTs for ``scale * base`` (external spins ``espin``) into ``dst``.

        Intermediates are spin-summed: X_s for a spin assignment of its free
        labels is the sum over the spins of the labels contracted at step s,
        so no spin term is evaluated twice.  Contributions that differ only
        by renaming summed labels are merged.  Returns the updated beta flag.
        """
        order = self._order(base)
        facs = [base[0]] + [base[k] for k in order]
        free = [list(facs[0][1])]
        shared = [[]]
        for s in range(1, len(facs)):
            prev = free[s - 1]
            tl = list(facs[s][1])
            sh = [l for l in prev if l in tl]
            shared.append(sh)
            free.append([l for l in prev if l not in sh] + [l for l in tl if l not in sh])
        last = len(facs) - 1
        memo = {}

        def get(s, spins):
            key = (s, tuple(sorted(spins.items())))
            if key in memo:
                return memo[key]
            if s == 0:
                r = map_factor(facs[0][0], facs[0][1], spins, undressed)
                out = [] if r is None else [(r[0], r[1])]
                memo[key] = out
                return out
            contribs = self._contribs(s, spins, facs, free, shared, get, undressed)
            if not contribs:
                memo[key] = []
                return []
            axes = [Axis(l, SIZE[(_sp(l), spins[l])]) for l in free[s]]
            name = self.new_x([a.size for a in axes])
            xv = View(name, axes)
            b = 0
            for alpha, xa, tb in contribs:
                self._gett(xv, xa, tb, alpha, b, tag)
                b = 1
            memo[key] = [(1, xv)]
            return memo[key]

        spins = {l: espin[l] for l in free[last]}
        nops, nx = len(self.ops), self.nx
        contribs = self._contribs(last, spins, facs, free, shared, get, undressed)
        if not contribs:
            # intermediates built for a product whose final contraction vanishes are dead
            del self.ops[nops:]
            for k in range(nx, self.nx):
                self.buffers.pop(f'X{k}', None)
            self.nx = nx
            return beta
        for alpha, xa, tb in contribs:
            self._gett(dst, xa, tb, alpha * float(scale), beta, tag)
            beta = 1
        return beta

    def _contribs(self, s, spins, facs, free, shared, get, undressed):
        sh = shared[s]
        prevfree = free[s - 1]
        merged = {}
        orderk = []
        for ds in itertools.product((0, 1), repeat=len(sh)):
            sp = dict(spins)
            sp.update(zip(sh, ds))
            r = map_factor(facs[s][0], facs[s][1], sp, undressed)
            if r is None:
                continue
            xs = get(s - 1, {l: sp[l] for l in prevfree})
            if not xs:
                continue
            st, tv = r
            for sx, xv in xs:
                ren = {}
                for a in xv.axes + tv.axes:
                    if a.label in sh and a.label not in ren:
                        ren[a.label] = f'k{len(ren)}'
                key = (xv.buf, tuple((ren.get(a.label, a.label), a.size, a.start) for a in xv.axes),
                       tv.buf, tuple((ren.get(a.label, a.label), a.size, a.start) for a in tv.axes))
                if key not in merged:
                    merged[key] = [0, xv, tv]
                    orderk.append(key)
                merged[key][0] += st * sx
        return [(merged[k][0], merged[k][1], merged[k][2]) for k in orderk if merged[k][0] != 0]

    def _gett(self, c, a, b, alpha, beta, tag):
        lsz = _label_size([a, b, c], self.sizes)
        f = 2
        for l in set(a.labels()) | set(b.labels()):
            f *= lsz[l]
        self.flops += f
        self.ops.append(Gett(c, a, b, float(alpha), beta, tag))

    @staticmethod
    def _z_order(labels, mem):
        """Axis order of a Z buffer: the assemble step reads Z once per permutation
        tau of its member list, so put last the Z labels that most permutations
        send to the target's last axes (those reads then walk Z contiguously)."""
        target = list(labels)               # target axis order i0.., a0..
        rest = list(labels)
        order = []
        for pos in reversed(range(len(target))):
            t = target[pos]
            best = max(rest, key=lambda l: (sum(1 for tau, _ in mem if tau[l] == t), -rest.index(l)))
            order.insert(0, best)
            rest.remove(best)
        return order

    # -- residual of one block -------------------------------------------------
    def emit_block(self, block, terms=None, undressed=False, mode='jacobi', defer=False):
        """GETTs of one block's residual and its closing ASSEMBLE.

        ``terms`` defaults to the CC residual of the block's level; ``defer``
        leaves out the PHASE marker and returns the ASSEMBLE instead of
        appending it (Jacobi updates that must follow every residual).
        """
        level = int(block[1])
        spins_t = block_spins(block)
        ext_o = [f'i{k}' for k in range(level)]
        ext_v = [f'a{k}' for k in range(level)]
        tspin = {l: s for l, s in zip(ext_o, spins_t)}
        tspin.update({l: s for l, s in zip(ext_v, spins_t)})
        if terms is None:
            terms = wick.residual_terms(level, self.tranks)
        groups = wick.orbit_groups(level, terms, workers=self.workers)
        asm = Assemble(block, mode)
        block_start = len(self.ops)
        direct = {}
        direct_order = []
        zshare = {}
        if not defer:
            self.ops.append(Simple('PHASE', (block,)))
        for gi, (base, members) in enumerate(groups):
            bypat = {}
            for tau, c in members:
                pat = tuple(tspin[tau[l]] for l in ext_o + ext_v)
                bypat.setdefault(pat, []).append((tau, c))
            for pat, mem in bypat.items():
                espin = dict(zip(ext_o + ext_v, pat))
                if len(base) == 1:
                    name, ls = base[0]
                    r = map_factor(name, ls, espin, undressed)
                    if r is None:
                        continue
                    sign, v = r
                    for tau, c in mem:
                        axes = [Axis(tau[a.label], a.size, a.start) for a in v.axes]
                        key = View(v.buf, axes).text()
                        if key not in direct:
                            direct[key] = [Fraction(0), View(v.buf, axes)]
                            direct_order.append(key)
                        direct[key][0] += c * sign
                    continue
                mem_sorted = sorted(mem, key=lambda tc: tuple(tc[0][l] for l in ext_o + ext_v))
                zaxes = [Axis(l, SIZE[(_sp(l), espin[l])]) for l in self._z_order(ext_o + ext_v, mem_sorted)]
                c0 = mem_sorted[0][1]
                norm = (pat, tuple((tuple(tc[0][l] for l in ext_o + ext_v), tc[1] / c0) for tc in mem_sorted))
                if norm in zshare:
                    z, cref, state = zshare[norm]
                    scale = c0 / cref
                    state[0] = self.emit_chain(base, espin, View(z, zaxes), scale, f'{block}.g{gi}', state[0],
                                               undressed)
                else:
                    nz, nx, nops = self.nz, self.nx, len(self.ops)
                    z = self.new_z([a.size for a in zaxes])
                    state = [0]
                    state[0] = self.emit_chain(base, espin, View(z, zaxes), Fraction(1), f'{block}.g{gi}', 0,
                                               undressed)
                    if state[0] == 0:
                        # every spin term of this group vanishes: no buffer, no assemble terms
                        assert len(self.ops) == nops
                        del self.buffers[z]
                        self.nz = nz
                        continue
                    zshare[norm] = (z, c0, state)
                    for tau, c in mem_sorted:
                        axes = [Axis(tau[a.label], a.size) for a in zaxes]
                        asm.terms.append((c, View(z, axes)))
        for key in direct_order:
            c, v = direct[key]
            if c != 0:
                asm.terms.append((c, v))
        self._restrict_block(block_start, asm)
        if defer:
            return asm
        self.ops.append(asm)

    def _op_groups(self, op, zl):
        grp = []
        for side in (op.a, op.b):
            for g in antisym_groups(side):
                gg = tuple(l for l in g if l in zl)
                if len(gg) >= 2:
                    grp.append(gg)
        return grp

    def _restrict_block(self, start, asm):
        """Antisymmetry restrictions for the GETTs of one block (ops[start:]).

        Contracted labels forming an antisymmetric group of both operands are
        summed over increasing tuples (the runtime scales alpha by the group's
        factorial).  A Z buffer is declared antisymmetric in the label groups
        that every contribution inherits from one operand; its GETTs then only
        produce increasing tuples and the assemble step reads Z sorted with sign.
        An expensive contribution that would lose its own restriction by sharing
        a Z with less symmetric ones gets a Z buffer of its own.
        """
        ops = self.ops[start:]
        byz = {}
        for op in ops:
            if isinstance(op, Gett) and op.c.buf.startswith('Z'):
                byz.setdefault(op.c.buf, []).append(op)

        def pairs(groups):
            return frozenset((a, b) for g in groups for a in g for b in g if a < b)

        for z in list(byz):
            gs = byz[z]
            zl = gs[0].c.labels()
            sigs = [pairs(self._op_groups(op, zl)) for op in gs]
            common = frozenset.intersection(*sigs)
            moved = {}
            for op, sg in zip(gs, sigs):
                m, n, k, _ = gett_count(op, self.sizes)
                if sg > common and 2 * m * n * k > 1e9:
                    moved.setdefault(sg, []).append(op)
            if not moved:
                continue
            zterms = [(c, v) for c, v in asm.terms if v.buf == z]
            keep = [op for op in gs if not any(op in lst for lst in moved.values())]
            for sg, lst in moved.items():
                nz = self.new_z(list(self.buffers[z][1]))
                for op in lst:
                    op.c = View(nz, op.c.axes)
                    op.beta = 1
                lst[0].beta = 0
                byz[nz] = lst
                for c, v in zterms:
                    asm.terms.append((c, View(nz, v.axes)))
            byz[z] = keep
            if keep:
                keep[0].beta = 0
            else:
                asm.terms[:] = [(c, v) for c, v in asm.terms if v.buf != z]
                del self.buffers[z]
                del byz[z]
        for z, gs in byz.items():
            zl = gs[0].c.labels()
            groups = _refine([self._op_groups(op, zl) for op in gs], zl)
            if groups:
                groups = [tuple(sorted(g, key=zl.index)) for g in groups]
                self.zgroups[z] = [tuple(zl.index(l) for l in g) for g in groups]
                for op in gs:
                    op.restrict = op.restrict + [list(g) for g in groups]
        for op in ops:
            if not isinstance(op, Gett):
                continue
            ka = antisym_groups(op.a)
            kb = antisym_groups(op.b)
            kl = set(op.a.labels()) & set(op.b.labels())
            for ga in ka:
                for gb in kb:
                    common = [l for l in ga if l in gb and l in kl]
                    if len(common) >= 2:
                        op.restrict = op.restrict + [common]

    def emit_dress(self):
        """exp(-T1) H exp(T1): copy undressed blocks, four quarter transforms each."""
        self.ops.append(Simple('PHASE', ('dress',)))
        for d, s in (('VAA', 'VAA0'), ('VAB', 'VAB0'), ('VBB', 'VBB0'), ('HA', 'HA0'), ('HB', 'HB0')):
            self.ops.append(Simple('COPY', (d, s)))
        full = lambda l: Axis(l, 'n')
        spins_of = {'VAA': (0, 0, 0, 0), 'VAB': (0, 1, 0, 1), 'VBB': (1, 1, 1, 1), 'HA': (0, 0), 'HB': (1, 1)}
        for buf, sps in spins_of.items():
            rank = len(sps)
            creators = [0, 1] if rank == 4 else [0]
            annih = [2, 3] if rank == 4 else [1]
            for slot in range(rank):
                sp = sps[slot]
                t1 = 'T1A' if sp == 0 else 'T1B'
                o, v = ('oa', 'va') if sp == 0 else ('ob', 'vb')
                rest = [f'x{k}' for k in range(rank)]
                if slot in creators:
                    # X[p in v] -= sum_i t1[i,p] X[p = i]
                    caxes = [full(l) for l in rest]
                    caxes[slot] = Axis('p', v, o)
                    baxes = [full(l) for l in rest]
                    baxes[slot] = Axis('i', o)
                    a = View(t1, [Axis('i', o), Axis('p', v)])
                    self.ops.append(Gett(View(buf, caxes), a, View(buf, baxes), -1.0, 1, 'dress'))
                else:
                    # X[r in o] += sum_a X[r = a] t1[r,a]
                    caxes = [full(l) for l in rest]
                    caxes[slot] = Axis('r', o)
                    baxes = [full(l) for l in rest]
                    baxes[slot] = Axis('e', v, o)
                    a = View(t1, [Axis('r', o), Axis('e', v)])
                    self.ops.append(Gett(View(buf, caxes), a, View(buf, baxes), 1.0, 1, 'dress'))
        # f = h + sum_i v[p,i,q,i]
        self.ops.append(Simple('COPY', ('FA', 'HA')))
        self.ops.append(Simple('COPY', ('FB', 'HB')))
        P, Q = Axis('p', 'n'), Axis('q', 'n')
        ia, ib = Axis('i', 'oa'), Axis('i', 'ob')
        self.ops.append(Gett(View('FA', [P, Q]), View('VAA', [P, ia, Q, ia]), View('ONES', [ia]), 1.0, 1, 'dress'))
        self.ops.append(Gett(View('FA', [P, Q]), View('VAB', [P, ib, Q, ib]), View('ONES', [ib]), 1.0, 1, 'dress'))
        self.ops.append(Gett(View('FB', [P, Q]), View('VBB', [P, ib, Q, ib]), View('ONES', [ib]), 1.0, 1, 'dress'))
        self.ops.append(Gett(View('FB', [P, Q]), View('VAB', [ia, P, ia, Q]), View('ONES', [ia]), 1.0, 1, 'dress'))

    def emit_energy(self):
        """E_cor with undressed f, v (``src/energy.f90:138-270``) into scalar E."""
        self.ops.append(Simple('PHASE', ('energy',)))
        self.ops.append(Simple('ZERO', ('E',)))
        for coef, tensors in wick.energy_terms():
            self.emit_chain(tensors, {}, View('E', []), coef, 'energy', 1, undressed=True)

    def emit_rhf_copy(self, block):
        src = {'T2C': 'T2A', 'T1B': 'T1A', 'T3D': 'T3A', 'T4E': 'T4A'}
        self.ops.append(Simple('PHASE', (block,)))
        level = int(block[1])
        lab = [f'i{k}' for k in range(level)] + [f'a{k}' for k in range(level)]
        dims = BLOCK_DIMS[block]
        if block in src:
            s = src[block]
            v = View(s, [Axis(l, d) for l, d in zip(lab, BLOCK_DIMS[s])])
        elif block == 'T3C':
            # T3C[i,j,k,a,b,c] = T3B[j,k,i,b,c,a]   (src/cc/tran3Bto3C.f90)
            order = ['i1', 'i2', 'i0', 'a1', 'a2', 'a0']
            v = View('T3B', [Axis(l, d) for l, d in zip(order, BLOCK_DIMS['T3B'])])
        elif block == 'T4D':
            order = ['i1', 'i2', 'i3', 'i0', 'a1', 'a2', 'a3', 'a0']
            v = View('T4B', [Axis(l, d) for l, d in zip(order, BLOCK_DIMS['T4B'])])
        else:
            raise KeyError(block)
        self.ops.append(Assemble(block, 'copy', [(Fraction(1), v)]))

    def build(self):
        n = 'n'
        for b in ('FA0', 'FB0', 'HA0', 'HB0', 'FA', 'FB', 'HA', 'HB'):
            self.buf(b, 'int', (n, n))
        for b in ('VAA0', 'VAB0', 'VBB0', 'VAA', 'VAB', 'VBB'):
            self.buf(b, 'int', (n, n, n, n))
        self.buf('ONES', 'ones', (n,))
        self.buf('E', 'scalar', ())
        for b, d in BLOCK_DIMS.items():
            if b[0] == 'T' and int(b[1]) <= max(3, self.nmax):
                self.buf(b, 'amp', d)
        order = ['T2A', 'T2C', 'T2B', 'T1A', 'T1B']
        if self.nmax >= 3:
            order += ['T3A', 'T3D', 'T3B', 'T3C']
        if self.nmax >= 4:
            order += ['T4A', 'T4B', 'T4C', 'T4D', 'T4E']
        self.emit_dress()
        for b in order:
            if b == 'T1B' and not self.rhf:
                self.emit_dress()
            if b == 'T3A':
                self.emit_dress()
            if self.rhf and b in ('T2C', 'T1B', 'T3D', 'T3C', 'T4D', 'T4E'):
                self.emit_rhf_copy(b)
            else:
                self.emit_block(b)
        self.emit_energy()
        merge_equal_views(self)
        return merge_shared_operand(self)

    def build_crcc(self):
        """CCSD sweep followed by the CR-CC(2,3) phases (``src/calc_driver.f90:55-73``).

        crcc     marker: ops before it form the CC sweep and energy
        dress    T1 dressing at the converged CCSD amplitudes
        CRDIAG   Hbar(CCSD) one- and two-body diagonals, three-body ``cal_d3`` sums
        lambda   every left residual LH (bare f, v; T1, T2, L1, L2), then the
                 Jacobi step of all five L blocks (``update_l2``): the residual
                 of every block is taken from the old lambda
        lenergy  sqrt(sum LH^2) + E_cor (``calculate_left_energy``)
        triplesX moments M3X and left projections L3X of spin block X, then
                 the four-denominator sums of ``crcc23`` into E23
        """
        from . import lagrange
        assert self.method == 'CCSD'
        self.build()
        n = 'n'
        for b in ('L1A', 'L1B', 'L2A', 'L2B', 'L2C'):
            self.buf(b, 'lamp', BLOCK_DIMS[b])
        for x in 'ABCD':
            self.buf('M3' + x, 'tri', BLOCK_DIMS['M3' + x])
            self.buf('L3' + x, 'tri', BLOCK_DIMS['L3' + x])
        for b in ('HDA', 'HDB'):
            self.buf(b, 'crd', (n,))
        for b in ('H2AA', 'H2AB', 'H2BB'):
            self.buf(b, 'crd', (n, n))
        for b in ('W1A', 'W1B', 'W1C', 'W1D', 'W2A', 'W2B', 'W2C', 'W2D'):
            self.buf(b, 'crd', (n, n, n))
        for b in ('LN', 'EL', 'ECOR'):
            self.buf(b, 'scalar', ())
        self.buf('E23', 'scalar', ('4',))
        self.ops.append(Simple('PHASE', ('crcc',)))
        self.emit_dress()
        self.ops.append(Simple('CRDIAG', ()))
        self.ops.append(Simple('PHASE', ('lambda',)))
        self.ops.append(Simple('ZERO', ('LN',)))
        lam_start = len(self.ops)
        asms = []
        self.lam_last = True
        for b in ('L1A', 'L1B', 'L2A', 'L2B', 'L2C'):
            terms = lagrange.left_residual_terms(int(b[1]))
            asms.append(self.emit_block(b, terms=terms, undressed=True, mode='ljacobi', defer=True))
        self.lam_last = False
        self._hoist_lambda_free(lam_start)
        self.ops += asms
        self.ops.append(Simple('PHASE', ('lenergy',)))
        self.ops.append(Simple('LENERGY', ()))
        for x in 'ABCD':
            self.ops.append(Simple('PHASE', ('triples' + x,)))
            self.ops.append(self.emit_block('M3' + x, terms=lagrange.triples_moment_terms(), mode='copy',
                                            defer=True))
            self.ops.append(self.emit_block('L3' + x, terms=lagrange.triples_left_terms(), mode='copy',
                                            defer=True))
            self.ops.append(Simple('CRCC', (x,)))
        return self

    def _hoist_lambda_free(self, start):
        """Move the intermediates of ops[start:] that do not depend on lambda ahead of
        the ``lambda`` phase marker (they are computed once per left solve) and
        give them dedicated buffers (kind ``hx``, names Y*)."""
        lam = {'L1A', 'L1B', 'L2A', 'L2B', 'L2C'}
        ops = self.ops[start:]
        dep = {}
        for op in ops:
            if isinstance(op, Gett) and op.c.buf.startswith('X'):
                d = op.a.buf in lam or op.b.buf in lam or dep.get(op.a.buf, False) or dep.get(op.b.buf, False)
                dep[op.c.buf] = dep.get(op.c.buf, False) or d
        hoist = {x for x, d in dep.items() if not d}
        ren = {}
        for x in sorted(hoist, key=lambda q: int(q[1:])):
            ren[x] = f'Y{len(ren)}'
            kind, dims = self.buffers.pop(x)
            self.buffers[ren[x]] = ('hx', dims)
        moved, kept = [], []
        for op in ops:
            if isinstance(op, Gett):
                for v in (op.a, op.b, op.c):
                    if v.buf in ren:
                        v.buf = ren[v.buf]
                (moved if op.c.buf.startswith('Y') else kept).append(op)
            else:
                kept.append(op)
        k = max(i for i in range(start) if isinstance(self.ops[i], Simple) and self.ops[i].kind == 'PHASE'
                and self.ops[i].args[0] == 'lambda')
        self.ops[k:] = moved + self.ops[k:start] + kept

    def text(self):
        lines = [f'PLAN {self.method} rhf={int(self.rhf)}']
        for name, (kind, dims) in self.buffers.items():
            g = ''
            if name in self.zgroups:
                g = ' G=' + ';'.join(','.join(str(a) for a in grp) for grp in self.zgroups[name])
            lines.append(f'BUF {name} {kind} {len(dims)} ' + ' '.join(dims) + g)
        lines.append(f'OPS {len(self.ops)}')
        for op in self.ops:
            lines.append(op.text())
        lines.append('END')
        return '\n'.join(lines) + '\n'


def build_plan(method, rhf=False, workers=None):
    if method == 'CR-CC(2,3)':
        b = PlanBuilder('CCSD', rhf, workers=workers).build_crcc()
        b.method = 'CR-CC(2,3)'
        return b
    return PlanBuilder(method, rhf, workers=workers).build()


def _choose(n, k):
    from math import comb
    return comb(n, k)


def gett_count(op, sizes=SIZES_C2):
    """(M, N, K, alpha scale) of a GETT after its antisymmetry restrictions."""
    lsz = _label_size([op.a, op.b, op.c], sizes)
    uniq = lambda ls: list(dict.fromkeys(ls))
    al, bl, cl = uniq(op.a.labels()), uniq(op.b.labels()), uniq(op.c.labels())
    ml = [l for l in al if l in cl]
    nl = [l for l in bl if l in cl]
    kl = [l for l in al if l in bl]
    out = []
    scale = 1
    for labs in (ml, nl, kl):
        rest = set(labs)
        cnt = 1
        for g in op.restrict:
            if set(g) <= set(labs):
                n = lsz[g[0]]
                cnt *= _choose(n, len(g))
                rest -= set(g)
                if labs is kl:
                    from math import factorial
                    scale *= factorial(len(g))
        for l in rest:
            cnt *= lsz[l]
        out.append(cnt)
    return out[0], out[1], out[2], scale


def plan_flops(builder, sizes=SIZES_C2):
    tot = 0
    for op in builder.ops:
        if isinstance(op, Gett):
            m, n, k, _ = gett_count(op, sizes)
            tot += 2 * m * n * k
    return tot


# ---------------------------------------------------------------------------
# Shared-operand merge.  Within one block phase, several GETTs often add into
# the same output view with the same amplitude operand, contracted over the
# same axes, and differ only in the small operand (an integral slice and a
# T2-built intermediate of the same shape: the linear ring term v T3 and the
# quadratic T2 v T3 term of the same topology, or f_oo T3 and X_oo T3).
# Z += a1 S1 T + a2 S2 T is then computed as W = a1 S1 + a2 S2 (a small
# buffer, built by GETTs against the scalar ONE) followed by one Z += W T, so
# the amplitude block is read once and the large product is done once.  The
# merged GETT takes the place of the group's last member (every small operand
# exists there; nothing reads Z before the block's assemble), and the first
# remaining writer of Z becomes the overwriting one.
# ---------------------------------------------------------------------------
_BIG = re.compile(r'^T[234][A-E]$')
_PHASE = re.compile(r'^T[1-4][A-E]$')


def merge_shared_operand(builder):
    ops = builder.ops
    phases = []
    start = None
    for i, op in enumerate(ops):
        if isinstance(op, Simple) and op.kind == 'PHASE':
            if start is not None:
                phases.append((start, i))
            start = i if _PHASE.match(str(op.args[0])) else None
    if start is not None:
        phases.append((start, len(ops)))
    if 'ONE' not in builder.buffers:
        builder.buf('ONE', 'ones', ())
    new_ops = list(ops)
    replace = {}    # op index -> list of ops in its place ([] deletes it)
    for p0, p1 in phases:
        groups = {}
        for i in range(p0 + 1, p1):
            op = ops[i]
            if not isinstance(op, Gett):
                continue
            for big_is_b in (True, False):
                big, small = (op.b, op.a) if big_is_b else (op.a, op.b)
                if not _BIG.match(big.buf) or _BIG.match(small.buf):
                    continue
                sl, bl, cl = small.labels(), big.labels(), op.c.labels()
                if len(set(sl)) != len(sl) or len(set(bl)) != len(bl):
                    continue
                kl = [l for l in bl if l not in cl]
                ren = {l: ('o' if _sp(l) == 'o' else 'v') + f'w{j}' for j, l in enumerate(kl)}
                outg = tuple(sorted(tuple(g) for g in op.restrict if all(l in cl for l in g)))
                kg = tuple(sorted(tuple(ren[l] for l in g) for g in op.restrict if all(l in ren for l in g)))
                if len(outg) + len(kg) != len(op.restrict):
                    continue
                bigc = View(big.buf, [Axis(ren.get(a.label, a.label), a.size, a.start) for a in big.axes])
                smallc = View(small.buf, [Axis(ren.get(a.label, a.label), a.size, a.start) for a in small.axes])
                key = (op.c.text(), bigc.text(), big_is_b, outg, kg)
                groups.setdefault(key, []).append((i, op, smallc, bigc))
                break
        used = set()
        for key, mem in groups.items():
            mem = [m for m in mem if m[0] not in used]
            if len(mem) < 2:
                continue
            c_text, big_text, big_is_b, outg, kg = key
            # one shape for W: the first member's small axes; every member's small view has the same labels
            wax = [Axis(a.label, a.size) for a in mem[0][2].axes]
            sig = sorted((a.label, a.size) for a in wax)
            if any(sorted((a.label, a.size) for a in m[2].axes) != sig for m in mem):
                continue
            w = builder.new_x([a.size for a in wax])
            wv = View(w, wax)
            seq = []
            for k, (i, op, smallc, bigc) in enumerate(mem):
                seq.append(Gett(wv, smallc, View('ONE', []), op.alpha, 0 if k == 0 else 1, op.tag))
            first = mem[0][1]
            a, b = (wv, mem[0][3]) if big_is_b else (mem[0][3], wv)
            seq.append(Gett(first.c, a, b, 1.0, 1, first.tag, [list(g) for g in outg] + [list(g) for g in kg]))
            for i, *_ in mem[:-1]:
                replace[i] = []
            replace[mem[-1][0]] = seq
            used.update(i for i, *_ in mem)
    if not replace:
        return builder
    out = []
    for i, op in enumerate(new_ops):
        out.extend(replace.get(i, [op]))
    builder.ops = out
    _first_writer_overwrites(builder)
    return builder


def _first_writer_overwrites(builder):
    """The first writer of every work buffer of a phase overwrites it, the others add."""
    seen = set()
    for op in builder.ops:
        if isinstance(op, Simple) and op.kind == 'PHASE':
            seen = set()
            continue
        if isinstance(op, Gett) and op.c.buf[0] in 'ZX':
            if op.c.buf not in seen:
                op.beta = 0
                seen.add(op.c.buf)
            else:
                op.beta = 1


# ---------------------------------------------------------------------------
# Equal-view merge.  The assemble of a block reads every Z buffer through a
# set of permuted views with coefficients.  Term groups of different topology
# often end with the same view set (up to one common factor) on Z buffers of
# the same shape and the same antisymmetric storage: the T3B residual has 25
# Z buffers but only 7 distinct (shape, storage, view set) classes.  The
# writers of every Z of a class then add into the class's first Z, scaled by
# the ratio of the view coefficients, and the assemble reads one buffer per
# class: fewer gathered terms per element, fewer buffers, and small-K writers
# of one Z view become one grouped launch in the runtime.
# ---------------------------------------------------------------------------
def merge_equal_views(builder):
    ops = builder.ops
    refs = {}
    for i, op in enumerate(ops):
        if isinstance(op, Gett):
            for role, v in (('c', op.c), ('a', op.a), ('b', op.b)):
                refs.setdefault(v.buf, []).append((i, role))
        elif isinstance(op, Assemble):
            for _, v in op.terms:
                refs.setdefault(v.buf, []).append((i, 'asm'))
            refs.setdefault(op.block, []).append((i, 'asm_out'))
        elif isinstance(op, Simple):
            for a in op.args:
                refs.setdefault(str(a), []).append((i, 'simple'))
    changed = False
    start = None
    for i, op in enumerate(ops):
        if isinstance(op, Simple) and op.kind == 'PHASE':
            start = i
            continue
        if not isinstance(op, Assemble) or start is None or not _PHASE.match(op.block):
            continue
        views = {}
        for c, v in op.terms:
            if v.buf.startswith('Z'):
                views.setdefault(v.buf, []).append((Fraction(c), tuple((a.label, a.size, a.start) for a in v.axes)))
        classes = {}
        for z, mem in views.items():
            # Z is written only by GETTs of this phase and read only by this assemble
            if not all((r == 'c' and start < j < i) or (j == i and r == 'asm') for j, r in refs.get(z, [])):
                continue
            mem = sorted(mem, key=lambda m: m[1])
            c0 = mem[0][0]
            key = (builder.buffers[z], tuple(builder.zgroups.get(z, ())), tuple((vk, c / c0) for c, vk in mem))
            classes.setdefault(key, []).append((z, c0))
        drop = {}
        for members in classes.values():
            (zt, ct), rest = members[0], members[1:]
            for z, c0 in rest:
                r = float(c0 / ct)
                for j, role in refs[z]:
                    if role == 'c':
                        w = ops[j]
                        w.c = View(zt, w.c.axes)
                        w.alpha = w.alpha * r
                drop[z] = zt
        if not drop:
            continue
        op.terms[:] = [(c, v) for c, v in op.terms if v.buf not in drop]
        for z in drop:
            del builder.buffers[z]
            builder.zgroups.pop(z, None)
        changed = True
    if changed:
        _first_writer_overwrites(builder)
    return builder
