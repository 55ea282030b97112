"""Many independent CC solves at once (64 CCSD Hamiltonians of uneven size).

Every Hamiltonian has its own context: its own stream, its own captured sweep
graph, its own DIIS ring.  Each iteration launches every active instance
(``ccq_b200_iterate_async``) before waiting for any (``ccq_b200_iterate_wait``),
so the kernels of different instances overlap on the device.  Each instance
follows the reference's ``jacobi_iter`` (``src/solve_cc.f90:175-269``) on its
own: iteration numbering, DIIS schedule, the three-|dE| convergence test and
the NaN / max-iteration exits, so its energy and iteration count are those of
a solve on its own.

Across GPUs the instances are independent units: ``shard`` assigns them to
ranks greedily by their o^2 v^4 cost (largest first, to the least loaded
rank); the only exchange is the host gather of the per-instance results.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import lib, synth

C3_COUNT = 64
C3_SEED = 1000


def c3_specs(count=C3_COUNT, seed=C3_SEED):
    """Instance i: norb ~ U{16..48} drawn from seed + i, nel = 2 floor(norb/5), L = 2 norb, sigma 0.03."""
    out = []
    for i in range(count):
        rng = np.random.default_rng(seed + i)
        n = int(rng.integers(16, 49))
        out.append(synth.SynthSpec(n, 2 * (n // 5), 2 * n, 0.03, seed + i))
    return out


def cost(spec):
    o = spec.nel // 2
    v = spec.norb - o
    return float(o) ** 2 * float(v) ** 4


def shard(specs, world):
    """Greedy longest-processing-time assignment: returns one index list per rank."""
    order = sorted(range(len(specs)), key=lambda i: -cost(specs[i]))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += cost(specs[i])
    return [sorted(p) for p in parts]


class Instance:
    def __init__(self, spec, calc_type='CCSD', diis_space=5, graph=True):
        t0 = time.perf_counter()
        s = synth.system(spec)
        d = s['dims']
        self.spec = spec
        t1 = time.perf_counter()
        self.ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, calc_type, s['f_a'], s['f_b'], s['v_aa'],
                               s['v_ab'], s['v_bb'], diis_space=diis_space)
        # host seconds spent generating the integrals and creating the context (threads overlap them)
        self.t_synth, self.t_ctx = t1 - t0, time.perf_counter() - t1
        # one stream per instance: the instances overlap one another, so each replays a
        # single-stream graph (mode 2) rather than its own concurrent one
        self.ctx.use_graph(2 if graph else 0)
        self.conv = [1.0, 1.0, 1.0]
        self.e = 0.0
        self.it = 0
        self.done = False
        self.failed = False
        self.device_ms = 0.0

    def step_launch(self):
        self.it += 1
        self.ctx.iterate_async(self.it)

    def step_finish(self, tol, max_iter):
        e_new, res, did = self.ctx.iterate_wait()
        self.device_ms += self.ctx.timing()[1]
        self.record(e_new, tol, max_iter)

    def record(self, e_new, tol, max_iter):
        """jacobi_iter's bookkeeping after iteration self.it: convergence, NaN and max_iter exits."""
        diff = self.e - e_new
        self.conv = [self.conv[1], self.conv[2], diff]
        self.e = e_new
        if all(abs(c) < tol for c in self.conv):
            self.done = True
        elif math.isnan(e_new):
            self.done = self.failed = True
        elif self.it == max_iter:
            self.done = self.failed = True

    def close(self):
        self.ctx.close()


def create_instances(specs, calc_type='CCSD', diis_space=5, graph=True, threads=None):
    """One context per spec, created by a pool of host threads (integral generation,
    plan instantiation and upload of different instances overlap) on the calling
    thread's CUDA device."""
    import os
    from concurrent.futures import ThreadPoolExecutor
    import torch
    dev = torch.cuda.current_device()

    def make(sp):
        torch.cuda.set_device(dev)
        return Instance(sp, calc_type, diis_space, graph)
    # four threads: more contend for the CUDA runtime's locks (64 contexts of 16-48 orbitals: 1.2 s with
    # four threads, 1.4 s with eight, 2.4 s with sixteen, 5.9 s with one)
    n = threads or min(4, os.cpu_count() or 1, max(1, len(specs)))
    if n <= 1 or len(specs) <= 1:
        return [make(sp) for sp in specs]
    with ThreadPoolExecutor(max_workers=n) as ex:
        return list(ex.map(make, specs))


def solve_pipelined(specs, tol=1e-8, max_iter=200, calc_type='CCSD', diis_space=5, threads=None):
    """Solve every instance, iterating the instances whose contexts exist while host threads create the others
    (largest first); returns (results, timings) as solve_batch, timings with ``total_s`` (first context
    requested to last instance converged) and ``setup_s`` (until the last context exists).  Each instance
    iterates exactly as on its own."""
    import os
    from concurrent.futures import ThreadPoolExecutor, FIRST_COMPLETED, wait
    import torch
    dev = torch.cuda.current_device()

    def make(sp):
        torch.cuda.set_device(dev)
        return Instance(sp, calc_type, diis_space, True)
    n = threads or min(4, os.cpu_count() or 1, max(1, len(specs)))
    order = sorted(range(len(specs)), key=lambda i: -cost(specs[i]))
    insts = [None] * len(specs)
    t0 = time.perf_counter()
    t_setup = t0
    active = []
    ex = ThreadPoolExecutor(max_workers=n)
    pending = {}
    try:
        pending = {ex.submit(make, specs[i]): i for i in order}
        while pending or active:
            if not active:
                wait(list(pending), return_when=FIRST_COMPLETED)
            for f in [f for f in pending if f.done()]:
                i = pending.pop(f)
                insts[i] = f.result()
                active.append(insts[i])
                if not pending:
                    t_setup = time.perf_counter()
            for x in active:
                x.step_launch()
            for x in active:
                x.step_finish(tol, max_iter)
            active = [x for x in active if not x.done]
        t2 = time.perf_counter()
        res = [dict(e_cor=x.e, iterations=x.it, failed=x.failed, device_ms=x.device_ms, synth_s=x.t_synth,
                    context_s=x.t_ctx) for x in insts]
    finally:
        ex.shutdown(wait=True)
        for f in pending:   # contexts still being created when an error stopped the loop
            if f.exception() is None:
                f.result().close()
        for x in insts:
            if x is not None:
                x.close()
    return res, {'setup_s': t_setup - t0, 'solve_s': t2 - t_setup, 'total_s': t2 - t0}


def solve_batch(specs, tol=1e-8, max_iter=200, calc_type='CCSD', diis_space=5, graph=True, t_init=None,
                keep_t=False, chunk=None, grouped=False):
    """Solve every instance; returns (results, timings).

    ``results[i]`` = dict(e_cor, iterations, failed, device_ms) (plus ``t``, the
    converged t_vec, with ``keep_t``); ``t_init[i]`` (a t_vec) replaces the
    T = 0 start of instance i.  Timings: wall seconds of context creation and
    of the iterations.  ``chunk`` bounds the number of contexts alive at once
    (the instances are solved in consecutive groups of that size).  ``grouped``:
    the instances iterate as one batch (``lib.Batch``): each plan operation of
    every active instance runs in one launch, then each instance's DIIS step.
    """
    if chunk and len(specs) > chunk:
        res, tim = [], {'setup_s': 0.0, 'solve_s': 0.0}
        for k in range(0, len(specs), chunk):
            r, t = solve_batch(specs[k:k + chunk], tol, max_iter, calc_type, diis_space, graph,
                               None if t_init is None else t_init[k:k + chunk], keep_t, grouped=grouped)
            res += r
            tim['setup_s'] += t['setup_s']
            tim['solve_s'] += t['solve_s']
        return res, tim
    t0 = time.perf_counter()
    insts = create_instances(specs, calc_type, diis_space, graph)
    if t_init is not None:
        for x, t in zip(insts, t_init):
            if t is not None:
                x.ctx.set_t(t)
    t1 = time.perf_counter()
    bt = None
    try:
        active = list(insts)
        if grouped:
            bt = lib.Batch([x.ctx for x in insts])
            it = 0
            while active:
                it += 1
                e, _, _ = bt.iterate(it, [0 if x.done else 1 for x in insts])
                ms = bt.stats()['sweep_ms'] / len(active)
                for j, x in enumerate(insts):
                    if not x.done:
                        x.it = it
                        x.device_ms += ms
                        x.record(float(e[j]), tol, max_iter)
                active = [x for x in active if not x.done]
        while active:
            for x in active:
                x.step_launch()
            for x in active:
                x.step_finish(tol, max_iter)
            active = [x for x in active if not x.done]
        t2 = time.perf_counter()
        res = [dict(e_cor=x.e, iterations=x.it, failed=x.failed, device_ms=x.device_ms, synth_s=x.t_synth,
                    context_s=x.t_ctx) for x in insts]
        if keep_t:
            for r, x in zip(res, insts):
                r['t'] = x.ctx.get_t()
    finally:
        if bt is not None:
            bt.close()
        for x in insts:
            x.close()
    return res, {'setup_s': t1 - t0, 'solve_s': t2 - t1}


def solve_sharded(specs, rank, world, gather, pipelined=False, **kw):
    """This rank's share of ``specs``; ``gather(obj)`` returns the list of every rank's obj."""
    parts = shard(specs, world)
    mine = parts[rank]
    run = solve_pipelined if pipelined else solve_batch
    empty = {'setup_s': 0.0, 'solve_s': 0.0, 'total_s': 0.0}
    res, tim = run([specs[i] for i in mine], **kw) if mine else ([], empty)
    allres = gather((mine, res, tim))
    out = [None] * len(specs)
    for idx, rr, _ in allres:
        for i, r in zip(idx, rr):
            out[i] = r
    return out, [t for _, _, t in allres]
