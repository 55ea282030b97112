"""Learned warm start over a family of Hamiltonians (lambda-swept off-diagonal ERIs).

The reference starts every solve from T = 0.  Here a new member of a family
whose other members are solved starts from a prediction:

  * base: the amplitudes of the two solved members that bracket its lambda,
    interpolated linearly in lambda (every T1, T2 and T3 element);
  * learned correction: two small networks (net2 for T2, net3 for T3,
    8 -> 32 -> 32 -> 1, tanh, FP32) predict each element's ratio to the base,
        t = t_int (1 + net(x)),
    from features that are symmetric under the amplitudes' antisymmetry (gap,
    occupied and virtual orbital-energy sums, log |t_int|, lambda, the two
    members' relative difference, the upper member's weight, and the weight
    w_lo w_hi (lambda_hi - lambda_lo)^2 of the interpolation's second-order
    error), so the start keeps every antisymmetry of the stored blocks.  The
    networks learn the curvature of t(lambda) that the interpolation misses:
    trained on the solved members, each predicted from its two neighbours,
    with elements drawn with probability proportional to t_int^2 so that the
    mean-squared loss weighs them as they weigh in the iteration's error.
T4 is built by the first sweep.  The exact CC iteration to the same tol
decides the result: the start only changes where the iteration begins, and
the plain T = 0 start is the fallback.

Training and inference run in this library's kernels (``ccq_b200_mlp_*``,
``csrc/mlp.cu``): forward, backward (mean-squared loss) and Adam, FP32.
Device memory comes from torch; every arithmetic step of the network is ours.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import integrals as I
from . import lib, synth

NFEAT = 8
C4_SEED = 4000
C4_COUNT = 200
C4_TRAIN = 150


def c4_family(norb=24, nel=10, count=C4_COUNT, seed=C4_SEED):
    """count Hamiltonians from one base seed, off-diagonal ERI scale lambda in [0.5, 2.0]."""
    lams = np.linspace(0.5, 2.0, count)
    return [synth.SynthSpec(norb, nel, 2 * norb, 0.03, seed, float(l)) for l in lams]


def c4_split(count=C4_COUNT, train=C4_TRAIN, seed=C4_SEED):
    perm = np.random.default_rng(seed).permutation(count)
    return sorted(perm[:train].tolist()), sorted(perm[train:].tolist())


def _bind():
    l = lib.load()
    for name, res, args in (
            ('ccq_b200_mlp_params', C.c_int, [C.c_int64]),
            ('ccq_b200_mlp_forward', C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                               C.c_void_p]),
            ('ccq_b200_mlp_grad', C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                            C.c_void_p, C.c_void_p]),
            ('ccq_b200_mlp_adam', C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_double,
                                            C.c_int64, C.c_void_p])):
        f = getattr(l, name)
        f.restype = res
        f.argtypes = args
    return l


def _check(code):
    if code != 0:
        raise lib.CCQB200Error(code, 'warm-start network kernel failed')


class WarmStart:
    """The network plus its feature / target standardisation."""

    def __init__(self, params=None, xmu=None, xsd=None, ysd=1.0, seed=0):
        self.l = _bind()
        self.np = self.l.ccq_b200_mlp_params(NFEAT)
        if self.np < 0:
            raise lib.CCQB200Error(self.np, 'bad feature count')
        if params is None:
            rng = np.random.default_rng(seed)
            H = 32
            p = []
            p.append(rng.normal(0, 1 / math.sqrt(NFEAT), (H, NFEAT)).ravel())
            p.append(np.zeros(H))
            p.append(rng.normal(0, 1 / math.sqrt(H), (H, H)).ravel())
            p.append(np.zeros(H))
            p.append(rng.normal(0, 1 / math.sqrt(H), H))
            p.append(np.zeros(1))
            params = np.concatenate(p)
        self.params = np.asarray(params, dtype=np.float32)
        assert self.params.size == self.np
        self.xmu = np.zeros(NFEAT) if xmu is None else np.asarray(xmu)
        self.xsd = np.ones(NFEAT) if xsd is None else np.asarray(xsd)
        self.ysd = float(ysd)

    def fit_scaling(self, X, y):
        self.xmu = X.mean(axis=0)
        self.xsd = X.std(axis=0) + 1e-12
        self.ysd = float(y.std() + 1e-12)

    # -- device steps -----------------------------------------------------------
    def train(self, X, y, epochs=400, batch=65536, lr=3e-3, seed=0, log=None):
        import torch
        dev = torch.device('cuda')
        Xs = torch.tensor(((X - self.xmu) / self.xsd).astype(np.float32), device=dev)
        ys = torch.tensor((y / self.ysd).astype(np.float32), device=dev)
        P = torch.tensor(self.params, device=dev)
        G = torch.zeros_like(P)
        M = torch.zeros_like(P)
        V = torch.zeros_like(P)
        loss = torch.zeros(1, dtype=torch.float32, device=dev)
        gen = torch.Generator(device=dev)
        gen.manual_seed(seed)
        n = Xs.shape[0]
        stream = torch.cuda.current_stream().cuda_stream
        hist = []
        step = 0
        for ep in range(epochs):
            idx = torch.randint(0, n, (min(batch, n),), device=dev, generator=gen)
            xb = Xs[idx].contiguous()
            yb = ys[idx].contiguous()
            step += 1
            _check(self.l.ccq_b200_mlp_grad(P.data_ptr(), NFEAT, xb.data_ptr(), yb.data_ptr(), xb.shape[0],
                                            G.data_ptr(), loss.data_ptr(), stream))
            _check(self.l.ccq_b200_mlp_adam(P.data_ptr(), G.data_ptr(), M.data_ptr(), V.data_ptr(), self.np, lr,
                                            step, stream))
            if ep % 50 == 0 or ep == epochs - 1:
                hist.append((ep, float(loss.item())))
                if log:
                    log(f'epoch {ep} loss {hist[-1][1]:.4e}')
        self.params = P.cpu().numpy()
        return hist

    def predict_ratio(self, X):
        import torch
        dev = torch.device('cuda')
        Xs = torch.tensor(((X - self.xmu) / self.xsd).astype(np.float32), device=dev)
        P = torch.tensor(self.params, device=dev)
        Y = torch.empty(Xs.shape[0], dtype=torch.float32, device=dev)
        _check(self.l.ccq_b200_mlp_forward(P.data_ptr(), NFEAT, Xs.data_ptr(), Xs.shape[0], Y.data_ptr(),
                                           torch.cuda.current_stream().cuda_stream))
        return Y.cpu().numpy().astype(np.float64) * self.ysd

    # -- persistence -------------------------------------------------------------
    def save(self, path):
        np.savez(path, params=self.params, xmu=self.xmu, xsd=self.xsd, ysd=self.ysd)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(z['params'], z['xmu'], z['xsd'], float(z['ysd']))


def mp2_t(s, layout):
    """t_vec with T2 = MP2, -<ij||ab> / (f_aa + f_bb - f_ii - f_jj) (the first sweep's result from T = 0),
    for comparison."""
    d = s['dims']
    fr = d.froz
    fa = np.diag(s['f_a'])[fr:]
    fb = np.diag(s['f_b'])[fr:]
    oa, ob = d.oa, d.ob
    t = np.zeros(layout.t_size)
    for name, (eo1, eo2, ev1, ev2, v) in (
            ('T2A', (fa[:oa], fa[:oa], fa[oa:], fa[oa:], s['v_aa'][:oa, :oa, oa:, oa:])),
            ('T2B', (fa[:oa], fb[:ob], fa[oa:], fb[ob:], s['v_ab'][:oa, :ob, oa:, ob:])),
            ('T2C', (fb[:ob], fb[:ob], fb[ob:], fb[ob:], s['v_bb'][:ob, :ob, ob:, ob:]))):
        gap = (ev1[None, None, :, None] + ev2[None, None, None, :] - eo1[:, None, None, None] -
               eo2[None, :, None, None])
        layout.view(t, name)[...] = -np.asarray(v) / gap
    return t


def tlayout(s):
    return I.TLayout(s['dims'])


def bracket(train_lams, lam, exclude=None):
    """Linear interpolation in lambda between solved family members: [(index, weight), ...].

    The nearest member below lam and the nearest above (``exclude`` left out);
    at an end of the family the two nearest on the one side (linear
    extrapolation); a single member when only one is left."""
    idx = [k for k in range(len(train_lams)) if k != exclude]
    lo = [k for k in idx if train_lams[k] <= lam]
    hi = [k for k in idx if train_lams[k] > lam]
    lo = sorted(lo, key=lambda k: (lam - train_lams[k], k))
    hi = sorted(hi, key=lambda k: (train_lams[k] - lam, k))
    if lo and hi:
        a, b = lo[0], hi[0]
    elif len(lo) >= 2:
        a, b = lo[0], lo[1]
    elif len(hi) >= 2:
        a, b = hi[0], hi[1]
    else:
        return [((lo or hi)[0], 1.0)]
    la, lb = train_lams[a], train_lams[b]
    wb = (lam - la) / (lb - la)
    return [(a, 1.0 - wb), (b, wb)]


def interp_start(s, lam, layout, members):
    """The base of the start, no network: members = [(weight, _, t_vec, lambda)] of ``bracket``;
    every amplitude (T1, T2, T3) interpolated linearly in lambda between the two members."""
    t = np.zeros(layout.t_size)
    for w, _, tv, la in members:
        t += w * np.asarray(tv)
    return t


# ---------------------------------------------------------------------------
# Two-anchor start with learned corrections to T2 and T3.
#
# The base is a linear interpolation in lambda between the two solved members
# that bracket the target (``bracket``), for every amplitude.  Two networks
# then correct it element by element,
#     T2 = t2_int (1 + net2(x)),   T3 = t3_int (1 + net3(x)),
# with features symmetric under the amplitudes' antisymmetry, so the start
# keeps every antisymmetry of the stored blocks.  The interpolation's error is
# mostly its second-order term, w_lo w_hi (lambda_hi - lambda_lo)^2 t''/2,
# so the features carry that weight, lambda and the two members' relative
# difference; the networks learn the curvature from the solved members.
# Without the networks (zero corrections) this is the ``interp`` start.
# ---------------------------------------------------------------------------
T2_BLOCKS = ('T2A', 'T2B', 'T2C')
T3_BLOCKS = ('T3A', 'T3B', 'T3C', 'T3D')


def _orbital_axes(s, shape_names):
    """Orbital energies along each axis of a stored block (names like 'oa', 'vb')."""
    d = s['dims']
    fr = d.froz
    fa = np.diag(s['f_a'])[fr:]
    fb = np.diag(s['f_b'])[fr:]
    ax = {'oa': fa[:d.oa], 'ob': fb[:d.ob], 'va': fa[d.oa:], 'vb': fb[d.ob:]}
    return [ax[n] for n in shape_names]


def _sum_axes(vecs, shape, first=0):
    """sum_k vecs[k] broadcast along axis first + k of an array of the given shape."""
    out = np.zeros(shape)
    for k, v in enumerate(vecs):
        out = out + v.reshape([-1 if j == first + k else 1 for j in range(len(shape))])
    return out


def _curvature_weight(members):
    """w_lo w_hi (lambda_hi - lambda_lo)^2: the factor of the interpolation's second-order error."""
    if len(members) < 2:
        return 0.0
    (w1, l1), (w2, l2) = [(m[0], m[3]) for m in members[:2]]
    return float(w1 * w2 * (l2 - l1) ** 2)


def interp_features(s, lam, members, layout, blocks, rng=None, per_block=None, cut=1e-3):
    """[(name, X [n, 8], base [n], sel, shape)] for the given blocks: base = the interpolated
    amplitudes (members = [(weight, anchor, t_vec, lambda)]) on the elements sel (|base| above
    cut * max |base|; with rng, per_block of them drawn with probability proportional to base^2, so
    that an unweighted mean-squared loss on the ratio weighs each element by its amplitude squared,
    the way the amplitudes enter the iteration's error).

    Features: gap, occupied and virtual energy sums, log |base|, lambda, the two members' relative
    difference (t_hi - t_lo) / base, the weight of the upper member and the curvature weight."""
    out = []
    hw = _curvature_weight(members)
    for name in blocks:
        shape = layout.shape[name]
        if not np.prod(shape):
            continue
        base = sum(w * np.asarray(layout.view(tv, name)).reshape(-1) for w, anc, tv, la in members)
        amax = np.abs(base).max()
        if amax == 0.0:
            continue
        sel = np.nonzero(np.abs(base) > cut * amax)[0]
        if rng is not None and per_block:
            w = base[sel] ** 2
            sel = np.sort(rng.choice(sel, per_block, replace=True, p=w / w.sum()))
        names = I.BLOCK_SHAPES[name]
        h = len(names) // 2
        ax = _orbital_axes(s, names)
        eo = _sum_axes(ax[:h], shape).reshape(-1)[sel]
        ev = _sum_axes(ax[h:], shape, h).reshape(-1)[sel]
        b = base[sel]
        if len(members) >= 2:
            lo, hi = sorted(members[:2], key=lambda m: m[3])
            d = (np.asarray(layout.view(hi[2], name)).reshape(-1)[sel] -
                 np.asarray(layout.view(lo[2], name)).reshape(-1)[sel]) / b
            whi = hi[0]
        else:
            d = np.zeros_like(b)
            whi = 1.0
        X = np.stack([ev - eo, eo, ev, np.log(np.abs(b)), np.full(b.shape, lam), np.clip(d, -4.0, 4.0),
                      np.full(b.shape, whi), np.full(b.shape, hw)], axis=-1)
        out.append((name, X, b, sel, shape))
    return out


class TwoAnchorWarmStart:
    """net2 (T2) and net3 (T3) over the interpolated start; trained and evaluated by the library's
    kernels (``ccq_b200_mlp_*``)."""

    def __init__(self, seed=0):
        self.net2 = WarmStart(seed=seed)
        self.net3 = WarmStart(seed=seed + 1)

    @staticmethod
    def samples(items, layout_of, per_block=20000, seed=0, cut=1e-3):
        """items = [(spec, t_vec (converged), members)]: (X2, y2, X3, y3) with targets t / base - 1
        clipped to [-0.5, 0.5], per_block elements per block and member drawn as in interp_features."""
        rng = np.random.default_rng(seed)
        xs = {2: [], 3: []}
        ys = {2: [], 3: []}
        for spec, tvec, members in items:
            s = synth.system(spec)
            lay = layout_of(s)
            for lvl, blocks in ((2, T2_BLOCKS), (3, T3_BLOCKS)):
                for name, X, b, sel, shape in interp_features(s, spec.lam, members, lay, blocks, rng, per_block,
                                                              cut):
                    t = np.asarray(lay.view(tvec, name)).reshape(-1)[sel]
                    xs[lvl].append(X)
                    ys[lvl].append(np.clip(t / b - 1.0, -0.5, 0.5))
        cat = lambda v, w: np.concatenate(v) if v else np.zeros(w)  # noqa: E731
        return cat(xs[2], (0, NFEAT)), cat(ys[2], 0), cat(xs[3], (0, NFEAT)), cat(ys[3], 0)

    def train(self, X2, y2, X3, y3, epochs=600, log=None):
        h2 = h3 = []
        if X2.shape[0]:
            self.net2.fit_scaling(X2, y2)
            h2 = self.net2.train(X2, y2, epochs=epochs, log=log)
        if X3.shape[0]:
            self.net3.fit_scaling(X3, y3)
            h3 = self.net3.train(X3, y3, epochs=epochs, log=log)
        return h2, h3

    def initial_t(self, s, lam, layout, members, use_t2=True, use_t3=True):
        """The interpolated t_vec with the networks' corrections on T2 (use_t2) and T3 (use_t3)."""
        t = interp_start(s, lam, layout, members)
        for use, net, blocks in ((use_t2, self.net2, T2_BLOCKS), (use_t3, self.net3, T3_BLOCKS)):
            if not use:
                continue
            for name, X, b, sel, shape in interp_features(s, lam, members, layout, blocks):
                v = layout.view(t, name).reshape(-1)
                v[sel] = b * (1.0 + np.clip(net.predict_ratio(X), -0.5, 0.5))
        return t


def study(method='CCSDT', norb=24, nel=10, count=C4_COUNT, train=C4_TRAIN, tol=1e-8, epochs=600, seed=C4_SEED,
          log=None, chunk=50):
    """The family solved plainly (T = 0, the reference's start), the networks trained on ``train`` of
    its members, and the other members solved from each start: iterations to tol and |dE| against the
    plain solves.

    Starts of the evaluation members: ``warm`` (interpolation in lambda between the two bracketing
    solved members, corrected by net2 on T2 and net3 on T3), and without a network: the T2 of MP2,
    the nearest solved member's amplitudes as they are (``anchor``), the interpolation alone
    (``interp``), and the networks on T2 only (``warm_t2_only``)."""
    import time
    from . import batch
    specs = [synth.SynthSpec(norb, nel, 2 * norb, 0.03, seed, float(l)) for l in np.linspace(0.5, 2.0, count)]
    tr, ev = c4_split(count, train, seed)
    t0 = time.perf_counter()
    plain, _ = batch.solve_batch(specs, tol=tol, calc_type=method, keep_t=True, chunk=chunk)
    t1 = time.perf_counter()
    tl = [specs[j].lam for j in tr]

    def members(i, exclude=None):
        return [(w, None, plain[tr[k]]['t'], specs[tr[k]].lam) for k, w in bracket(tl, specs[i].lam, exclude)]
    # training: every training member from its two bracketing neighbours (itself left out)
    items = [(specs[i], plain[i]['t'], members(i, k)) for k, i in enumerate(tr)]
    two = TwoAnchorWarmStart(seed=seed)
    X2, Y2, X3, Y3 = two.samples(items, tlayout, seed=seed)
    h2, h3 = two.train(X2, Y2, X3, Y3, epochs=epochs, log=log)
    t2 = time.perf_counter()
    starts = {'warm': [], 'mp2': [], 'anchor': [], 'interp': [], 'warm_t2_only': []}
    for i in ev:
        s = synth.system(specs[i])
        lay = tlayout(s)
        mem = members(i)
        starts['warm'].append(two.initial_t(s, specs[i].lam, lay, mem))
        starts['mp2'].append(mp2_t(s, lay))
        near = min(tr, key=lambda j: (abs(specs[j].lam - specs[i].lam), j))
        starts['anchor'].append(np.array(plain[near]['t']))
        starts['interp'].append(interp_start(s, specs[i].lam, lay, mem))
        starts['warm_t2_only'].append(two.initial_t(s, specs[i].lam, lay, mem, use_t3=False))
    t3 = time.perf_counter()
    legs = {}
    for name, st in starts.items():
        rr, _ = batch.solve_batch([specs[i] for i in ev], tol=tol, calc_type=method, t_init=st, chunk=chunk)
        it_ = np.array([r['iterations'] for r in rr], dtype=float)
        legs[name] = {'iterations_mean': float(it_.mean()),
                      'max_dE': float(max(abs(plain[i]['e_cor'] - r['e_cor']) for i, r in zip(ev, rr))),
                      'failed': int(sum(r['failed'] for r in rr))}
        if name == 'warm':
            t4 = time.perf_counter()
    pi = np.array([plain[i]['iterations'] for i in ev], dtype=float)
    w = legs['warm']
    return {'method': method, 'norb': norb, 'nel': nel, 'family': count, 'train': len(tr), 'eval': len(ev),
            'tol': tol, 'plain_iterations_mean': float(pi.mean()), 'warm_iterations_mean': w['iterations_mean'],
            'iteration_reduction': float(1.0 - w['iterations_mean'] / pi.mean()), 'max_dE': w['max_dE'],
            'failed': int(w['failed'] + sum(plain[i]['failed'] for i in ev)),
            'starts': {k: v for k, v in legs.items()},
            'network_gain_over_interp': float(1.0 - w['iterations_mean'] / legs['interp']['iterations_mean']),
            'train_samples': {'t2': int(X2.shape[0]), 't3': int(X3.shape[0])},
            'loss': {'t2': [h2[0][1], h2[-1][1]] if h2 else None, 't3': [h3[0][1], h3[-1][1]] if h3 else None},
            'loss_history': {'t2': h2, 't3': h3},
            'seconds': {'plain_family': t1 - t0, 'train': t2 - t1, 'starts': t3 - t2, 'warm_eval': t4 - t3}}
