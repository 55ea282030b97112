"""numpy emulation of libccq_b200's plan semantics (test helper).

Reproduces what the C++ runtime does with a plan, not what the equations
mean: offset tables built label by label, restriction groups enumerated for
increasing tuples with alpha scaled by the group factorial, Z buffers read
sorted-with-sign by the assemble step, orbit permutations written from
canonical elements.  Work buffers start as NaN, so any read of an element
that no operation wrote poisons the result.
"""
import itertools

import numpy as np

from oracle import solver as S


def _table(labels, ext, strides, groups):
    gidx = []
    for g in groups:
        pos = [labels.index(l) for l in g if l in labels]
        if len(pos) == len(g):
            gidx.append(pos)
    out = []
    for idx in itertools.product(*[range(ext[l]) for l in labels]):
        if all(idx[g[q]] > idx[g[q - 1]] for g in gidx for q in range(1, len(g))):
            out.append([sum(i * st[l] for i, l in zip(idx, labels)) for st in strides])
    if not labels:
        out = [[0 for _ in strides]]
    return np.array(out, dtype=np.int64).reshape(-1, len(strides))


def _perm_sign(p):
    s = 1
    for x in range(len(p)):
        for y in range(x + 1, len(p)):
            if p[y] < p[x]:
                s = -s
    return s


def emulate(bc, tvec, ops):
    sizes = bc.sizes
    bufs = bc.plan['buffers']

    def arr(name):
        return bc._array(name, tvec)

    def resolve(v):
        name, axes = v
        a = arr(name)
        strides = [s // 8 for s in a.strides]
        off, st, ext, order = 0, {}, {}, []
        for d, (lab, size, start) in enumerate(axes):
            off += sizes[start] * strides[d]
            if lab not in st:
                st[lab], ext[lab] = 0, sizes[size]
                order.append(lab)
            st[lab] += strides[d]
        return a.reshape(-1), off, st, ext, order, strides

    for op in ops:
        kind = op[0]
        if kind == 'GETT':
            _, alpha, beta, cv, av, bv, tag, restrict = op
            Cf, co, cst, cext, cord, _ = resolve(cv)
            Af, ao, ast, aext, aord, _ = resolve(av)
            Bf, bo, bst, bext, bord, _ = resolve(bv)
            ml = [l for l in aord if l in cst and l not in bst]
            kl = [l for l in aord if l in bst and l not in cst]
            nl = [l for l in bord if l in cst and l not in ast]
            ext = {**aext, **bext}
            scale = 1.0
            for g in restrict:
                if all(l in kl for l in g):
                    scale *= float(np.prod(range(1, len(g) + 1)))
                else:
                    assert all(l in ml for l in g) or all(l in nl for l in g), (g, ml, nl)
            tm = _table(ml, ext, [ast, cst], restrict)
            tn = _table(nl, ext, [bst, cst], restrict)
            tk = _table(kl, ext, [ast, bst], restrict)
            Am = Af[ao + tm[:, 0][:, None] + tk[:, 0][None, :]]
            Bm = Bf[bo + tn[:, 0][:, None] + tk[:, 1][None, :]]
            Cm = alpha * scale * (Am @ Bm.T)
            idx = co + tm[:, 1][:, None] + tn[:, 1][None, :]
            assert len(np.unique(idx)) == idx.size
            if beta:
                Cf[idx] += Cm
            else:
                Cf[idx] = Cm
        elif kind == 'ASSEMBLE':
            _, block, mode, terms = op
            T = arr(block)
            Tf = T.reshape(-1)
            level = int(block[1])
            rank = 2 * level
            target = [f'i{k}' for k in range(level)] + [f'a{k}' for k in range(level)]
            spins = S.block_spins(block)
            tst = [s // 8 for s in T.strides]
            runs = []
            for half in range(2):
                d = half * level
                while d < (half + 1) * level:
                    e = d + 1
                    while e < (half + 1) * level and spins[e % level] == spins[d % level]:
                        e += 1
                    runs.append(list(range(d, e)))
                    d = e
            perms = []
            for combo in itertools.product(*[list(itertools.permutations(range(len(r)))) for r in runs]):
                P = [0] * rank
                sg = 1
                for r, p in zip(runs, combo):
                    sg *= _perm_sign(p)
                    for q in range(len(r)):
                        P[r[q]] = r[p[q]]
                perms.append((P, sg))
            tt = []
            for coef, v in terms:
                Vf, vo, vst, vext, vord, vstrides = resolve(v)
                src = [target.index(a[0]) for a in v[1]]
                groups = bufs[v[0]][2] if len(bufs[v[0]]) > 2 else []
                tt.append((coef, Vf, vo, vstrides, src, groups))
            fa, fb = bc.fdiag_a, bc.fdiag_b
            nocc = [bc.dims.oa, bc.dims.ob]
            new = {}
            for x in itertools.product(*[range(s) for s in T.shape]):
                if any(not ((d % level == 0) or spins[d % level] != spins[d % level - 1]) and x[d] <= x[d - 1]
                       for d in range(1, rank)):
                    continue
                R = 0.0
                for coef, Vf, vo, vstrides, src, groups in tt:
                    y = [x[s] for s in src]
                    sg = 1
                    zero = False
                    for g in groups:
                        vals = [y[j] for j in g]
                        order = sorted(range(len(vals)), key=lambda q: vals[q])
                        sg *= _perm_sign(order)
                        sv = [vals[q] for q in order]
                        if len(set(sv)) != len(sv):
                            zero = True
                        for j, val in zip(g, sv):
                            y[j] = val
                    if zero:
                        continue
                    R += sg * coef * Vf[vo + sum(a * b for a, b in zip(vstrides, y))]
                toff = sum(a * b for a, b in zip(tst, x))
                if mode == 'jacobi':
                    D = bc.shift
                    for d in range(level):
                        D -= (fa if spins[d] == 0 else fb)[x[d]]
                    for d in range(level, rank):
                        sp = spins[d - level]
                        D += (fa if sp == 0 else fb)[nocc[sp] + x[d]]
                    tn = Tf[toff] - R / D
                else:
                    tn = R
                for P, sg in perms:
                    new[sum(tst[d] * x[P[d]] for d in range(rank))] = sg * tn
            for o, val in new.items():
                Tf[o] = val
        elif kind == 'COPY':
            bc.buf[op[1]][...] = bc.buf[op[2]]
        elif kind == 'ZERO':
            arr(op[1])[...] = 0.0


def parse_annotated(text):
    """Plan text with the R= / G= annotations kept (oracle/blockcc drops them)."""
    from oracle.blockcc import parse_view
    lines = text.strip().split('\n')
    plan = {'buffers': {}, 'ops': []}
    k = 1
    while lines[k].startswith('BUF'):
        p = lines[k].split()
        nd = int(p[3])
        groups = []
        if len(p) > 4 + nd and p[4 + nd].startswith('G='):
            groups = [[int(a) for a in g.split(',')] for g in p[4 + nd][2:].split(';')]
        plan['buffers'][p[1]] = (p[2], p[4:4 + nd], groups)
        k += 1
    k += 1
    while lines[k] != 'END':
        p = lines[k].split()
        if p[0] == 'GETT':
            tag, restrict = '', []
            for w in p[6:]:
                if w.startswith('R='):
                    restrict = [g.split(',') for g in w[2:].split(';')]
                else:
                    tag = w
            plan['ops'].append(('GETT', float(p[1]), int(p[2]), parse_view(p[3]), parse_view(p[4]),
                                parse_view(p[5]), tag, restrict))
            k += 1
        elif p[0] == 'ASSEMBLE':
            nt = int(p[3])
            terms = [(float(lines[k + 1 + j].split()[1]), parse_view(lines[k + 1 + j].split()[2])) for j in range(nt)]
            plan['ops'].append(('ASSEMBLE', p[1], p[2], terms))
            k += 1 + nt
        else:
            plan['ops'].append(tuple(p))
            k += 1
    return plan
