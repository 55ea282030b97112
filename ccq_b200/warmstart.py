"""Learned warm start of the T2 amplitudes (lambda-swept Hamiltonian family).

The reference starts every solve from T = 0, so its first sweep produces the
MP2 doubles t = -<ij||ab> / D (D = f_aa + f_bb - f_ii - f_jj).  Here a small
network predicts the remaining correction per amplitude,

    t2_init = mp2 * (1 + r),   r = net(features)

where the features are symmetric under the antisymmetry of the amplitude
(gap D, the occupied and virtual orbital-energy sums, log |mp2|, log |v|, the
family parameter lambda, and, from the nearest solved member of the family
(the anchor), its converged ratio t/mp2 - 1 at the same element and the lambda
distance to it), so t2_init keeps the antisymmetry of mp2 and vanishes where
mp2 does.  T1 and T3 start from the anchor's converged values (zero without an
anchor); T4 is built by the first sweep.  The exact CC iteration to the same
tol decides the result: the warm start only changes where the iteration starts.

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


def block_features(fdiag_o, fdiag_v, v_block, lam, anchor_ratio=None, dlam=0.0):
    """Features and MP2 amplitudes of one stored T2 block.

    fdiag_o = (occ energies of the two occupied axes), fdiag_v likewise;
    v_block[i, j, a, b] = <ij||ab> in the block's spin pattern; anchor_ratio =
    the anchor's converged t/mp2 - 1 on this block (zero without an anchor),
    dlam = lambda - the anchor's lambda.
    Returns (X [N, NFEAT], mp2 [N]) over every stored element, and the block shape.
    """
    eo1, eo2 = fdiag_o
    ev1, ev2 = fdiag_v
    eo = eo1[:, None, None, None] + eo2[None, :, None, None]
    ev = ev1[None, None, :, None] + ev2[None, None, None, :]
    gap = ev - eo
    mp2 = -v_block / gap
    shape = v_block.shape
    tiny = 1e-300
    ar = np.zeros(shape) if anchor_ratio is None else np.asarray(anchor_ratio).reshape(shape)
    X = np.stack([gap, np.broadcast_to(eo, shape), np.broadcast_to(ev, shape),
                  np.log(np.abs(mp2) + tiny), np.log(np.abs(v_block) + tiny),
                  np.full(shape, lam), ar, np.full(shape, dlam)], axis=-1).reshape(-1, NFEAT)
    return X, mp2.reshape(-1), shape


def ratios(mp2, t, cut=1e-6):
    """t / mp2 - 1 where |mp2| exceeds cut * max |mp2| (else 0), clipped to [-2, 2]."""
    r = np.zeros_like(mp2)
    m = np.abs(mp2) > cut * np.abs(mp2).max()
    r[m] = np.clip((t[m] - mp2[m]) / mp2[m], -2.0, 2.0)
    return r


def anchor_of(spec, t):
    """(lambda, {block: converged t/mp2 - 1}) of a solved family member (t: its t_vec)."""
    s = synth.system(spec)
    lay = tlayout(s)
    out = {}
    for name, X, mp2, shape in system_blocks(s, spec.lam):
        out[name] = ratios(mp2, np.asarray(lay.view(t, name)).reshape(-1)).reshape(shape)
    return spec.lam, out


def system_blocks(s, lam, anchor=None):
    """(name, X, mp2, shape) for T2A, T2B, T2C of a system from ``synth.system``;
    anchor = ``anchor_of`` of the nearest solved family member, or None."""
    d = s['dims']
    fr = d.froz
    fa = np.diag(s['f_a'])[fr:]
    fb = np.diag(s['f_b'])[fr:]
    oa, ob = d.oa, d.ob
    vaa, vab, vbb = s['v_aa'], s['v_ab'], s['v_bb']
    out = []
    for name, (eoa, eob, eva, evb, v) in (
            ('T2A', (fa[:oa], fa[:oa], fa[oa:], fa[oa:], vaa[:oa, :oa, oa:, oa:])),
            ('T2B', (fa[:oa], fb[:ob], fa[oa:], fb[ob:], vab[:oa, :ob, oa:, ob:])),
            ('T2C', (fb[:ob], fb[:ob], fb[ob:], fb[ob:], vbb[:ob, :ob, ob:, ob:]))):
        ar = None if anchor is None else anchor[1][name]
        dl = 0.0 if anchor is None else lam - anchor[0]
        X, mp2, shape = block_features((eoa, eob), (eva, evb), np.asarray(v), lam, ar, dl)
        out.append((name, X, mp2, shape))
    return out


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

    # -- data -------------------------------------------------------------------
    @staticmethod
    def samples(specs_and_t2, cut=1e-6):
        """Training samples from (spec, {block: converged T2 array}, anchor) triples.

        Target r = (t - mp2) / mp2 on elements whose |mp2| exceeds cut * max|mp2|,
        clipped to [-2, 2].
        """
        xs, ys = [], []
        for spec, t2, anchor in specs_and_t2:
            s = synth.system(spec)
            for name, X, mp2, shape in system_blocks(s, spec.lam, anchor):
                t = np.asarray(t2[name]).reshape(-1)
                m = np.abs(mp2) > cut * np.abs(mp2).max()
                r = np.clip((t[m] - mp2[m]) / mp2[m], -2.0, 2.0)
                xs.append(X[m])
                ys.append(r)
        return np.concatenate(xs), np.concatenate(ys)

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

    def initial_t(self, s, lam, layout, anchor=None, t_anchor=None):
        """A full t_vec (reference layout): T2 = mp2 (1 + r); T1 and T3 from the anchor's
        converged t_vec ``t_anchor`` when given, else zero."""
        t = np.zeros(layout.t_size) if t_anchor is None else np.array(t_anchor, dtype=np.float64)
        for name, X, mp2, shape in system_blocks(s, lam, anchor):
            r = np.clip(self.predict_ratio(X), -2.0, 2.0)
            layout.view(t, name)[...] = (mp2 * (1.0 + r)).reshape(shape)
        return t

    # -- persistence -------------------------------------------------------------
    def save(self, path):
        np.savez(path, params=self.params, xmu=self.xmu, xsd=self.xsd, ysd=self.ysd)

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(z['params'], z['xmu'], z['xsd'], float(z['ysd']))


def mp2_t(s, layout):
    """t_vec with T2 = MP2 (the first sweep's result from T = 0), for comparison."""
    t = np.zeros(layout.t_size)
    for name, X, mp2, shape in system_blocks(s, 1.0):
        layout.view(t, name)[...] = mp2.reshape(shape)
    return t


def tlayout(s):
    return I.TLayout(s['dims'])


def study(method='CCSDT', norb=24, nel=10, count=C4_COUNT, train=C4_TRAIN, tol=1e-8, epochs=600, seed=C4_SEED,
          log=None):
    """Plain solves of the whole family, training on ``train`` of them, warm-started
    solves of the rest; iterations to tol and |dE| between the two starts."""
    import time
    from . import batch
    specs = [synth.SynthSpec(norb, nel, 2 * norb, 0.03, seed, float(l)) for l in np.linspace(0.5, 2.0, count)]
    tr, ev = c4_split(count, train, seed)
    t0 = time.perf_counter()
    plain, _ = batch.solve_batch(specs, tol=tol, calc_type=method, keep_t=True)
    t1 = time.perf_counter()
    anchors = {i: anchor_of(specs[i], plain[i]['t']) for i in tr}

    def nearest(i, exclude_self):
        # the solved training member closest in lambda (another one for a training member)
        cand = [j for j in tr if not (exclude_self and j == i)]
        return min(cand, key=lambda j: (abs(specs[j].lam - specs[i].lam), j))
    data = []
    for i in tr:
        s = synth.system(specs[i])
        lay = tlayout(s)
        data.append((specs[i], {b: lay.view(plain[i]['t'], b) for b in ('T2A', 'T2B', 'T2C')},
                     anchors[nearest(i, True)]))
    X, y = WarmStart.samples(data)
    ws = WarmStart(seed=seed)
    ws.fit_scaling(X, y)
    hist = ws.train(X, y, epochs=epochs, log=log)
    t2 = time.perf_counter()
    inits, mp2s = [], []
    for i in ev:
        s = synth.system(specs[i])
        lay = tlayout(s)
        a = nearest(i, False)
        inits.append(ws.initial_t(s, specs[i].lam, lay, anchors[a], plain[a]['t']))
        mp2s.append(mp2_t(s, lay))
    warm, _ = batch.solve_batch([specs[i] for i in ev], tol=tol, calc_type=method, t_init=inits)
    t3 = time.perf_counter()
    mp2r, _ = batch.solve_batch([specs[i] for i in ev], tol=tol, calc_type=method, t_init=mp2s)
    pi = np.array([plain[i]['iterations'] for i in ev], dtype=float)
    wi = np.array([r['iterations'] for r in warm], dtype=float)
    mi = np.array([r['iterations'] for r in mp2r], dtype=float)
    de = max(abs(plain[i]['e_cor'] - r['e_cor']) for i, r in zip(ev, warm))
    return {'method': method, 'norb': norb, 'nel': nel, 'family': count, 'train': len(tr), 'eval': len(ev),
            'tol': tol, 'plain_iterations_mean': float(pi.mean()), 'warm_iterations_mean': float(wi.mean()),
            'mp2_start_iterations_mean': float(mi.mean()),
            'iteration_reduction': float(1.0 - wi.sum() / pi.sum()), 'max_dE': float(de),
            'failed': int(sum(r['failed'] for r in warm) + sum(plain[i]['failed'] for i in ev)),
            'train_samples': int(X.shape[0]), 'loss_history': hist,
            'seconds': {'plain_family': t1 - t0, 'train': t2 - t1, 'warm_eval': t3 - t2}}
