"""Benchmark: CCSDT iteration on 40 spatial orbitals (16 electrons, 64 virtual spin orbitals).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision split|fp64]

A step is one CC iteration of ccq's solver loop (update sweep of every T1..T3
spin block in the reference's order, energy, DIIS ring write, residuum, and
the DIIS extrapolation every diis_space+1 iterations) on the seeded synthetic
Hamiltonian (ERIs from an L=80 factorisation, sigma=0.025, seed 2; no molecular
integrals travel with the repository).  The working set (T3 blocks 4 x 134 MB
plus the DIIS ring) exceeds the 126 MB L2, so no flush is needed between steps.

``value`` is device seconds per iteration (CUDA events on the library's
stream), whole job: max over ranks of the time / (ranks x K).  Multi-GPU runs
are independent replicas (one solve per GPU, no collective on the data path).
``e2e`` is the same metric through the C ABI with the T vector in pinned host
memory: every step reads it from the host and writes it back
(ccq_b200_iterate_host: the T3 blocks are read at their canonical elements
inside the sweep, each operation waiting only for the blocks it reads, and
every block is copied out as soon as the sweep has written it).  ``--impl reference`` times the CPU
executor of this repository's CCSDT plan (numpy + threaded BLAS) on this host
(ccq itself cannot be built: no Fortran compiler).

Besides the headline legs (FP64 and split, each autotuned first), the line
carries the convergence of the headline path to tol against the FP64 oracle
fixture, CR-CC(2,3) at 32 orbitals, 64 batched CCSD solves (sharded over the
ranks) and the learned warm start on a 200-member CCSDT family; --no-crcc,
--no-batch, --no-warmstart, --no-converge, --no-tune skip them.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = 'CCSDT s/iter + TFLOP/s on 1 B200, split vs FP64 GPU; |dE| vs FP64 oracle'
WORKLOAD = 'CCSDT, 40 spatial orbitals, nel=16, nvir=64, L=80, sigma=0.025, seed=2, UHF spin blocks'
L2_NOTE = 'working set (T3 4x134 MB + DIIS ring) > 126 MB L2, no flush'


def parse():
    p = argparse.ArgumentParser()
    p.add_argument('--gpus', type=int, default=1)
    p.add_argument('--steps', type=int, default=40)
    p.add_argument('--warmup', type=int, default=3)
    p.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    p.add_argument('--precision', default='auto', choices=['auto', 'split', 'fp64'])
    p.add_argument('--slices', type=int, default=int(os.environ.get('CCQ_B200_SLICES', '4')))
    p.add_argument('--no-cpu-baseline', action='store_true')
    p.add_argument('--no-converge', action='store_true')
    p.add_argument('--no-peaks', action='store_true', help='use MEASURED_PEAKS.json / fallback only')
    p.add_argument('--no-tune', action='store_true', help='keep the shape heuristics (no autotuning sweep)')
    p.add_argument('--no-crcc', action='store_true', help='skip the CR-CC(2,3) leg (32 orbitals)')
    p.add_argument('--no-batch', action='store_true', help='skip the batched CCSD leg (64 Hamiltonians)')
    p.add_argument('--no-ccsdt', action='store_true', help='skip the active-space CCSDt leg (40 orbitals)')
    p.add_argument('--no-warmstart', action='store_true',
                   help='skip the learned warm-start study (200 CCSDT Hamiltonians at 24 orbitals, about 40 s)')
    return p.parse_args()


def dist_init(n):
    import torch
    rank = int(os.environ.get('RANK', '0'))
    world = int(os.environ.get('WORLD_SIZE', '1'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(x, world):
    """Max of a per-rank device time over all ranks (the whole job waits for the slowest replica)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_seconds_per_iter(ms_total_rank, world, steps):
    """Whole-job s/iter of independent replicas: slowest rank's time over all iterations of all ranks."""
    return allmax(ms_total_rank, world) / 1e3 / (world * steps)


class Clocks:
    """nvidia-smi samples every 50 ms; the summary keeps the samples taken inside the timed window."""
    FIELDS = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,'
              'clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,'
              'clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap')

    def __init__(self, local):
        self.local = local
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f'ccq_b200_clocks_rank{local}_{os.getpid()}.csv')
        self.stamps = []   # (host time, line count) when the timed window opens and closes

    def start(self):
        """Starts sampling (before the warm-up, so that the sampler runs when the timed window opens)."""
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.local), f'--query-gpu={self.FIELDS}',
                                          '--format=csv,noheader,nounits', '-lms', '50'],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def mark(self):
        """Opens or closes the timed window: the number of samples written so far."""
        try:
            self.fh.flush()
            with open(self.path) as fh:
                self.stamps.append(sum(1 for _ in fh))
        except Exception:
            self.stamps.append(None)

    def stop(self):
        if not self.proc:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['nvidia-smi unavailable']}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        lines = open(self.path).readlines()
        try:
            os.remove(self.path)
        except OSError:
            pass
        window = 'timed region'
        if len(self.stamps) == 2 and None not in self.stamps and self.stamps[1] > self.stamps[0]:
            lines = lines[self.stamps[0]:self.stamps[1]]
        else:
            window = 'warm-up and timed region'
        for line in lines:
            f = [x.strip() for x in line.split(',')]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith('active'):
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': ['no samples']}
        return {'sm_mhz': float(np.median(sm)), 'sm_max_mhz': max(smax), 'reasons': sorted(reasons),
                'samples': len(sm), 'window': window}


def measure_peaks():
    """cuBLAS DGEMM and int8 GEMM throughput on this GPU (denominators not in MEASURED_PEAKS.json)."""
    import torch
    out = {}
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device='cuda')
    b = torch.randn(n, n, dtype=torch.float64, device='cuda')
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    out['fp64_tflops'] = 2 * n ** 3 / (best * 1e-3) / 1e12
    del a, b
    try:
        a = torch.randint(-64, 64, (n, n), dtype=torch.int8, device='cuda')
        b = torch.randint(-64, 64, (n, n), dtype=torch.int8, device='cuda').t().contiguous().t()
        for _ in range(2):
            torch._int_mm(a, b)
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch._int_mm(a, b)
            e.record()
            torch.cuda.synchronize()
            best = min(best, s.elapsed_time(e))
        out['int8_tops'] = 2 * n ** 3 / (best * 1e-3) / 1e12
    except Exception as ex:  # noqa: BLE001
        out['int8_tops'] = None
        out['int8_error'] = str(ex)[:120]
    torch.cuda.empty_cache()
    return out


def measured_peaks_file():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        return json.load(open(p)), 'measured'
    return {'hbm_gbs': 6650.0, 'bf16_tflops': 1590.0, 'bf16_tflops_sustained': 1400.0}, 'fallback'


def golden_c2():
    p = os.path.join(ROOT, 'tests', 'golden', 'synthetic.json')
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get('c2_ccsdt')
    return None


# FLOPs of one CCSDT iteration of the reference's own algorithm at 40 orbitals (o = 8, v = 32 per
# spin): a static count over its egemm calls (2 k1 k2 k3 with the i1, i2, i3 set before each call)
# and its explicit OpenMP loop bodies over the unique triples (2 per product term per inner
# iteration) in src/cc/t1A..t3D_update.f90: GEMMs 4.8e10 + T3 loops 1.62e11.  This engine's plan
# counts its own FLOPs from its GETT tables (flops_per_iter: 1.91e11 at this size).
REFERENCE_FLOPS_C2 = 2.10e11

# DRAM bytes (read + write) per gett_f64 launch in one tuned split-precision sweep of this workload,
# from one ncu capture of every GETT launch of that sweep (dram__bytes_read.sum + dram__bytes_write.sum,
# a single-pass metric set, full size): 17.0 GB over 527 launches of the 64x64, skinny, register-direct and
# small-K families.  Command: `ncu --nvtx --nvtx-include "sweep/" --metrics
# dram__bytes_read.sum,dram__bytes_write.sum,gpu__time_duration.sum --clock-control none --csv
# python bench.py --case sweep split /tmp/ops_split.txt 3 tune`.
GETT_F64_TRAFFIC = 32.18e6
GETT_F64_TRAFFIC_NOTE = ('traffic = DRAM bytes per gett_f64 launch (mean over the 527 launches of one tuned split '
                         'sweep, ncu dram__bytes_read.sum + dram__bytes_write.sum, captured at full size)')

BASELINE_KIND = ('numpy executor of this repository\'s CCSDT contraction plan (oracle/blockcc.py, threaded '
                 'BLAS); ccq itself cannot be built here or on the GPU box (no Fortran compiler)')


def cpu_reference(system, steps, warmup, budget_s=150.0):
    """The oracle port on this host's cores: oracle/blockcc.py executing the CCSDT plan in numpy.

    This is the repository's own formulation run on the CPU, not ccq's Fortran diagram code (which no
    compiler here can build); it is a reported baseline, not the reference's own speed."""
    from oracle.blockcc import BlockCC
    try:
        from threadpoolctl import threadpool_info
        cores = max([x.get('num_threads', 1) for x in threadpool_info()] or [os.cpu_count()])
    except Exception:  # noqa: BLE001
        cores = os.cpu_count()
    txt = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CCSDT.plan')).read()
    s = system
    bc = BlockCC(txt, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], s['dims'], 'CCSDT')
    from oracle import solver as S
    from ccq_b200 import integrals as I
    lay = I.TLayout(s['dims'])
    tvec = np.zeros(lay.t_size)
    ring = S.Ring(5, lay.t_size)
    times = []
    t_start = time.time()
    it = 0
    while True:
        it += 1
        t0 = time.perf_counter()
        bc.update(tvec)
        e = bc.energy(tvec)
        ring.write(it, tvec)
        ring.residuum(it)
        if it % 6 == 0:
            tvec[:] = ring.diis()
        dt = time.perf_counter() - t0
        if it > warmup:
            times.append(dt)
        if len(times) >= steps or (time.time() - t_start > budget_s and times):
            break
    return {'s_per_iter': float(np.median(times)), 'iters_timed': len(times), 'cores': int(cores or 1),
            'e_last': e}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from ccq_b200 import synth
    s = synth.system(synth.C2)
    w = max(0, min(args.warmup, 1))
    r = cpu_reference(s, max(1, min(args.steps, 3)), w)
    line = {
        'metric': METRIC, 'impl': 'reference', 'value': r['s_per_iter'], 'unit': 's/iter',
        'n_gpus': args.gpus, 'steps': r['iters_timed'], 'warmup': w, 'ms_per_step': r['s_per_iter'] * 1e3,
        'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64',
        'data': 'synthetic (seeded generator, no molecular integrals)',
        'config': {'workload': WORKLOAD, 'parallelism': f'replicas x{world}', 'l2': L2_NOTE},
        'threads': 'all host threads (threaded BLAS)',
        'cpu_baseline': {'value': r['s_per_iter'], 'unit': 's/iter', 'cores': r['cores'], 'kind': 'port',
                         'sample': f"{r['iters_timed']} full CCSDT iteration(s) after {w} warm-up; " + BASELINE_KIND},
        'e2e': {'value': r['s_per_iter'], 'unit': 's/iter', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0},
    }
    print(json.dumps(line), flush=True)


def golden(name):
    p = os.path.join(ROOT, 'tests', 'golden', 'synthetic.json')
    if not os.path.exists(p):
        return None
    return json.load(open(p)).get(name)


def crcc_leg(cpu_sample=True):
    """CR-CC(2,3) on the 32-orbital system (nel=14, nvir=50, L=64, sigma=0.03, seed=1).

    The whole calculation of ``calc_type=CR-CC(2,3)``: CCSD to tol 1e-10, the
    left CCSD solve to the same tol, and the four corrections; device times per
    phase (CUDA events on the library's stream) and the wall time of the
    complete call sequence.  The CPU sample times one CCSD iteration, one left
    iteration and the corrections with the numpy executor of the same plan.
    """
    from ccq_b200 import config, driver, lib, synth
    s = synth.system(synth.C1)
    d = s['dims']
    cfg = config.Config(calc_type='CR-CC(2,3)', tol=1e-10, diis_space=5, max_iter=200).calc_macros()
    t0 = time.perf_counter()
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CR-CC(2,3)', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                      s['v_bb'], diis_space=5)
    ctx.use_graph(True)
    r = driver.solve_cc(ctx, cfg, out=lambda x: None)
    cc_ms = sum(h['ms'] for h in r.history)
    ctx.lambda_init(r.e_cor)
    lms, en, conv, itl = [], 0.0, [1.0, 1.0, 1.0], 0
    for itl in range(1, cfg.max_iter + 1):
        e_new, res, did = ctx.lambda_iterate(itl)
        lms.append(ctx.timing()[1])
        conv = [conv[1], conv[2], en - e_new]
        en = e_new
        if all(abs(c) < cfg.tol for c in conv):
            break
    e23 = ctx.crcc23()
    tri_ms = ctx.timing()[0]
    wall = time.perf_counter() - t0
    lstat = ctx.stats()
    ctx.close()
    g = golden('c1_crcc23')
    out = {'workload': 'CR-CC(2,3), 32 spatial orbitals, nel=14, nvir=50, L=64, sigma=0.03, seed=1, UHF spin blocks',
           'wall_s': wall, 'ccsd_iterations': r.iterations, 'ccsd_device_ms': cc_ms,
           'left_iterations': itl, 'left_device_ms': float(sum(lms)), 'left_ms_per_iter': float(np.mean(lms)),
           'triples_device_ms': tri_ms, 'e_ccsd': r.e_cor, 'e23': [float(x) for x in e23],
           'dE23_vs_oracle': ([abs(a - b) for a, b in zip(e23, g['e23'])] if g else None),
           'dE_ccsd_vs_oracle': (abs(r.e_cor - g['e_cor']) if g else None),
           'iterations_match_oracle': ((r.iterations, itl) == (g['iterations'], g['left_iterations']) if g else None),
           'oracle': 'tests/golden/synthetic.json c1_crcc23 (numpy executor of the same plan)' if g else None}
    if cpu_sample:
        from oracle.blockcc import BlockCRCC
        text = open(os.path.join(ROOT, 'ccq_b200', 'plans', 'CRCC23.plan')).read()
        bc = BlockCRCC(text, s['f_a'], s['f_b'], s['v_aa'], s['v_ab'], s['v_bb'], d)
        tvec = np.zeros(bc.layout.t_size)
        t1 = time.perf_counter()
        bc.update(tvec)
        bc.energy(tvec)
        t_cc = time.perf_counter() - t1
        bc.lambda_init(tvec, -0.1)
        t1 = time.perf_counter()
        bc.lambda_update(bc.lvec, tvec)
        bc.lambda_energy(bc.lvec, tvec)
        t_l = time.perf_counter() - t1
        t1 = time.perf_counter()
        bc.crcc23(tvec)
        t_t = time.perf_counter() - t1
        est = t_cc * r.iterations + t_l * itl + t_t
        out['cpu_baseline'] = {'value': est, 'unit': 's per CR-CC(2,3) calculation (estimated)', 'cores': os.cpu_count(),
                               'kind': 'port', 'sample': f'one CCSD iteration ({t_cc:.2f} s), one left iteration '
                               f'({t_l:.2f} s) and the corrections ({t_t:.2f} s) with the numpy executor, scaled by '
                               f'the GPU run\'s iteration counts'}
    return out


def ccsdt_active_leg(s, steps=10, warmup=3, act_occ=2, act_unocc=6):
    """Active-space CCSDt on the 40-orbital CCSDT workload (act_occ = 2, act_unocc = 6: ccq's
    act_occ_b = occ_b - 2, act_unocc_a = occ_a + 6): the T3 residual contractions run over the active
    triples only.  FP64, graph replay, CUDA events per iteration (median)."""
    from ccq_b200 import lib
    d = s['dims']
    act = (d.occ_b - act_occ, d.occ_a + act_unocc)
    ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDt', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                      s['v_bb'], active=act)
    ctx.use_graph(True)
    it = 1
    for _ in range(warmup):
        ctx.iterate(it)
        it += 1
    ms = []
    for _ in range(steps):
        ctx.iterate(it)
        ms.append(ctx.timing()[1])
        it += 1
    st = ctx.stats()
    ctx.close()
    return {'workload': f'CCSDt, 40 spatial orbitals, act_occ={act_occ}, act_unocc={act_unocc} '
                        f'(act_occ_b={act[0]}, act_unocc_a={act[1]}), FP64',
            's_per_iter': float(np.median(ms)) / 1e3, 'flops_per_iter': st['flops'],
            'launches_per_iter': st['launches'], 'iterations_timed': steps}


def batch_leg(rank, world):
    """64 CCSD Hamiltonians of 16-48 spatial orbitals to tol 1e-8 (ccq_b200.batch.c3_specs).

    Instances are sharded over the ranks (no collective on the data path; a host
    gather of the results).  solves/s = 64 / the slowest rank's wall time of the
    iterations; context creation (integral upload, plan instantiation) is
    reported beside it.
    """
    from ccq_b200 import batch

    def gather(obj):
        if world == 1:
            return [obj]
        import torch.distributed as dist
        objs = [None] * world
        dist.all_gather_object(objs, obj)
        return objs
    specs = batch.c3_specs()
    g = golden('c3_batched_ccsd')
    legs = {}
    for name, grouped, piped in (('grouped', True, False), ('streams', False, False), ('pipelined', False, True)):
        barrier(world)
        res, tims = batch.solve_sharded(specs, rank, world, gather, pipelined=piped, tol=1e-8,
                                        **({} if piped else {'grouped': grouped}))
        solve_s = max(t['solve_s'] for t in tims)
        setup_s = max(t['setup_s'] for t in tims)
        total_s = max(t.get('total_s', t['setup_s'] + t['solve_s']) for t in tims)
        de = it_ok = None
        if g:
            de = max(abs(r['e_cor'] - x['e_cor']) for r, x in zip(res, g['instances']))
            it_ok = sum(r['iterations'] == x['iterations'] for r, x in zip(res, g['instances']))
        legs[name] = {'solves_per_s': len(specs) / solve_s, 'solve_wall_s': solve_s, 'setup_wall_s': setup_s,
                      'total_wall_s': total_s, 'e2e_solves_per_s': len(specs) / total_s,
                      'failed': sum(r['failed'] for r in res), 'max_dE_vs_oracle': de,
                      'iterations_match_oracle': it_ok}
        if piped:
            # iterations overlap the context creation: only the wall from start to the last solve means anything
            legs[name]['solves_per_s'] = None
            legs[name]['solve_wall_s'] = None
    # headline: one captured graph per instance on its own stream (the faster of the two here: the
    # batched CCSD sweep is bound by the T1 re-dressing of every instance's n^4 integrals, not by launches);
    # end to end, the pipelined run (instances iterate while the other contexts are being created)
    head = legs['streams']
    solve_s, setup_s = head['solve_wall_s'], head['setup_wall_s']
    de, it_ok = head['max_dE_vs_oracle'], head['iterations_match_oracle']
    return {'workload': '64 x CCSD, norb ~ U{16..48} (seed 1000+i), nel = 2 floor(norb/5), L = 2 norb, sigma 0.03, '
                        'tol 1e-8', 'solves_per_s': len(specs) / solve_s, 'solve_wall_s': solve_s,
            'setup_wall_s': setup_s,
            'e2e_solves_per_s': max(legs['pipelined']['e2e_solves_per_s'], head['e2e_solves_per_s']),
            'e2e_mode': 'pipelined' if legs['pipelined']['e2e_solves_per_s'] >= head['e2e_solves_per_s'] else 'streams',
            'setup_thread_s': {'integrals': sum(r['synth_s'] for r in res),
                               'contexts': sum(r['context_s'] for r in res)},
            'mode': 'streams (headline): one captured graph per instance on its own stream; grouped: each plan '
                    'operation of all instances in one launch (ccq_b200_batch_iterate); pipelined: streams, the '
                    'instances iterating while host threads create the remaining contexts (largest first)',
            'legs': legs,
            'failed': sum(r['failed'] for r in res), 'iterations_total': sum(r['iterations'] for r in res),
            'device_ms_sum': sum(r['device_ms'] for r in res),
            'max_dE_vs_oracle': de, 'iterations_match_oracle': it_ok,
            'oracle': 'tests/golden/synthetic.json c3_batched_ccsd (numpy executor, each instance alone)' if g else None,
            'cpu_oracle_seconds': g['seconds'] if g else None}


def time_leg(ctx, it0, steps, world):
    """Run `steps` iterations; returns (device ms list, energies)."""
    import torch
    ms, es = [], []
    barrier(world)
    torch.cuda.synchronize()
    for k in range(steps):
        e, res, did = ctx.iterate(it0 + k)
        ms.append(ctx.timing()[1])
        es.append(e)
    torch.cuda.synchronize()
    barrier(world)
    return ms, es


# ---------------------------------------------------------------------------
# single-kernel and single-sweep cases for profiler captures (small device footprint):
#   python bench.py --case egemm K1 K2 K3 [repeats]
#   python bench.py --case egemm_split K1 K2 K3 [slices] [tile|persistent]
#   python bench.py --case sweep fp64|split OUTFILE [warm-up iterations] [0|1|2|3|tune]
#   python bench.py --case warmstart CCSDT|CCSDTQ NORB NEL [COUNT TRAIN EPOCHS]
# egemm runs ccq_b200_egemm (the FP64 GETT kernel) on random column-major operands; the vvvv
# ladder of the CCSDT T3 update at 40 orbitals is (1024, 16384, 1024).
# ---------------------------------------------------------------------------
def run_case(argv):
    from ccq_b200 import lib
    kind = argv[0]
    if kind == 'egemm':
        k1, k2, k3 = (int(x) for x in argv[1:4])
        rep = int(argv[4]) if len(argv) > 4 else 1
        rng = np.random.default_rng(0)
        A = np.asfortranarray(rng.normal(size=(k3, k1)))
        B = np.asfortranarray(rng.normal(size=(k3, k2)))
        for _ in range(rep):
            t0 = time.perf_counter()
            C = lib.egemm(k1, k2, k3, A, B)
            dt = time.perf_counter() - t0
        ref = B[:, :64].T @ A[:, :64]
        err = float(np.abs(C[:64, :64] - ref).max())
        print(f'egemm {k1}x{k2}x{k3}: wall {dt * 1e3:.2f} ms (incl. copies), max err {err:.2e}')
        assert err < 1e-9
    elif kind == 'egemm_split':
        k1, k2, k3 = (int(x) for x in argv[1:4])
        S = int(argv[4]) if len(argv) > 4 else 4
        persistent = (argv[5] == 'persistent') if len(argv) > 5 else None
        rng = np.random.default_rng(0)
        A = np.asfortranarray(rng.normal(size=(k3, k1)))
        B = np.asfortranarray(rng.normal(size=(k3, k2)))
        for _ in range(3 if persistent is not None else 1):
            C = lib.egemm_split(k1, k2, k3, A, B, S, persistent=persistent)
        ref = B[:, :64].T @ A[:, :64]
        err = float(np.abs(C[:64, :64] - ref).max())
        # the split bound: 2^(-7S+2) k3 max|A| max|B|
        bound = 2.0 ** (-7 * S + 2) * k3 * np.abs(A[:, :64]).max() * np.abs(B[:, :64]).max()
        print(f'egemm_split {k1}x{k2}x{k3} S={S}: max err {err:.2e} (bound {bound:.2e})')
        assert err <= bound
    elif kind == 'sweep':
        # per-operation device times of one CCSDT sweep on the 40-orbital workload
        import os
        from ccq_b200 import synth
        prec = argv[1] if len(argv) > 1 else 'fp64'
        out = argv[2] if len(argv) > 2 else 'ops_profile.txt'
        warm = int(argv[3]) if len(argv) > 3 else 3
        family = argv[4] if len(argv) > 4 else '0'   # kernel family to force (0..3) or 'tune'
        s = synth.system(synth.C2)
        d = s['dims']
        # a one-vector DIIS ring keeps the device footprint small for profiler captures
        ctx = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                          s['v_bb'], diis_space=1)
        ctx.set_precision(lib.PREC_SPLIT if prec == 'split' else lib.PREC_FP64, 4)
        if family == 'tune':
            print('autotune (ms before, after):', ctx.autotune(3))
        elif family != '0':
            ctx.force_tile(int(family))
        for it in range(1, warm + 1):
            ctx.iterate(it)
        if os.path.exists(out):
            os.remove(out)
        os.environ['CCQ_B200_PROFILE_DUMP'] = out
        ctx.profile(True)
        import torch
        torch.cuda.synchronize()
        # an NVTX range around the profiled sweep: `ncu --nvtx --nvtx-include "sweep/"` captures its launches only
        torch.cuda.nvtx.range_push('sweep')
        ctx.iterate(warm + 1)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(ctx.profile_get())
        ctx.close()
    elif kind == 'warmstart':
        # the learned warm start on a lambda-swept family: METHOD NORB NEL [COUNT TRAIN EPOCHS]
        import json
        from ccq_b200 import warmstart
        method, norb, nel = argv[1], int(argv[2]), int(argv[3])
        count = int(argv[4]) if len(argv) > 4 else 200
        train = int(argv[5]) if len(argv) > 5 else 150
        epochs = int(argv[6]) if len(argv) > 6 else 600
        r = warmstart.study(method, norb, nel, count, train, epochs=epochs, log=print)
        print(json.dumps(r))
    else:
        raise SystemExit(f'unknown case {kind}')



def main():
    if len(sys.argv) > 2 and sys.argv[1] == '--case':
        return run_case(sys.argv[2:])
    args = parse()
    import torch
    rank, world, local = dist_init(args.gpus)
    if args.impl == 'reference':
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    from ccq_b200 import lib, synth
    # at least one DIIS cycle of warm-up (diis_space + 1 = 6 iterations): a context's first DIIS step pays
    # one-time costs (34-1229 ms were seen in the FP64 leg's timed window, 16 ms in isolated runs); the
    # line reports the warm-up actually done
    if args.warmup < 6:
        args.warmup = 6
    s = synth.system(synth.C2)
    d = s['dims']
    peaks_file, peaks_kind = measured_peaks_file()
    peaks_live = measure_peaks() if not args.no_peaks else {'fp64_tflops': 35.5, 'int8_tops': 3063.0,
                                                            'note': 'not measured (--no-peaks)'}

    def new_ctx():
        c = lib.Context(d.froz, d.occ_a, d.occ_b, d.orbs, 'CCSDT', s['f_a'], s['f_b'], s['v_aa'], s['v_ab'],
                        s['v_bb'], rhf=False, shift=0.0, diis_space=5)
        c.use_graph(True)
        return c

    ctx = new_ctx()
    split_ok = True
    try:
        ctx.set_precision(lib.PREC_SPLIT, args.slices)
        ctx.set_precision(lib.PREC_FP64, args.slices)
    except lib.CCQB200Error:
        split_ok = False
    headline = args.precision if args.precision != 'auto' else ('split' if split_ok else 'fp64')
    legs = ['fp64'] + (['split'] if split_ok and args.precision != 'fp64' else [])
    clocks = Clocks(local)
    results = {}
    tuning = {}
    it = 1
    for leg in legs:
        ctx.set_precision(lib.PREC_SPLIT if leg == 'split' else lib.PREC_FP64, args.slices)
        if not args.no_tune:
            # one eager sweep timing every contraction's candidates; amplitudes untouched
            t0 = time.perf_counter()
            before, after = ctx.autotune(3)
            tuning[leg] = {'gett_ms_heuristic': before, 'gett_ms_tuned': after,
                           'wall_s': time.perf_counter() - t0}
        if leg == headline:
            clocks.start()
        # warm-up continues the same solve (iterations keep counting, DIIS on schedule)
        for _ in range(args.warmup):
            ctx.iterate(it)
            it += 1
        if leg == headline:
            clocks.mark()
        ms, es = time_leg(ctx, it, args.steps, world)
        if leg == headline:
            clocks.mark()
            clk = clocks.stop()
        it += args.steps
        st = ctx.stats()
        tot = allmax(sum(ms), world)
        results[leg] = {'s_per_iter': job_seconds_per_iter(sum(ms), world, args.steps), 'ms_total': tot,
                        'ms_each': [round(x, 3) for x in ms],
                        'tflops': st['flops'] * world * args.steps / (tot * 1e-3) / 1e12,
                        'launches_per_iter': st['launches'], 'flops_per_iter': st['flops']}
    head = results[headline]

    # per-kernel roofline: eager sweep with events around every launch (and every launch's shape in a dump)
    ctx.set_precision(lib.PREC_SPLIT if headline == 'split' else lib.PREC_FP64, args.slices)
    dump = os.path.join(tempfile.gettempdir(), f'ccq_b200_ops_rank{rank}_{os.getpid()}.txt')
    if os.path.exists(dump):
        os.remove(dump)
    os.environ['CCQ_B200_PROFILE_DUMP'] = dump
    ctx.profile(True)
    for _ in range(2):
        ctx.iterate(it)
        it += 1
    prof = ctx.profile_get()
    ctx.profile(False)
    del os.environ['CCQ_B200_PROFILE_DUMP']
    # dominant kernel of the headline leg = largest share of device time
    kname = max(('gett_f64', 'gett_split', 'assemble'), key=lambda k: prof[k]['ms'])
    per_sweep = {k: {'ms': v['ms'] / 2, 'launches': v['launches'] // 2, 'flops': v['flops'] / 2}
                 for k, v in prof.items()}
    tot_ms = sum(v['ms'] for v in prof.values())
    shares = {k: v['ms'] / tot_ms for k, v in prof.items()} if tot_ms else {}
    slices = args.slices
    fp64_peak = peaks_live['fp64_tflops']
    int8_peak = peaks_live.get('int8_tops') or 2 * peaks_file['bf16_tflops']

    def gett_line(k):
        p_ = prof[k]
        if p_['ms'] <= 0:
            return None
        if k == 'gett_f64':
            a = p_['flops'] / (p_['ms'] * 1e-3) / 1e12
            return {'bound': 'tensor', 'achieved': a, 'peak': fp64_peak, 'unit': 'TFLOP/s', 'frac': a / fp64_peak,
                    'peak_source': 'cuBLAS DGEMM 8192^3 measured in this run (of measured)'}
        # split: int8 products actually issued = S(S+1)/2 per FP64-algorithmic multiply-add
        a = p_['flops'] * slices * (slices + 1) / 2 / (p_['ms'] * 1e-3) / 1e12
        return {'bound': 'tensor', 'achieved': a, 'peak': int8_peak, 'unit': 'TOP/s (int8)', 'frac': a / int8_peak,
                'peak_source': 'cuBLASLt int8 GEMM 8192^3 measured in this run (of measured)',
                'fp64_equivalent_tflops': p_['flops'] / (p_['ms'] * 1e-3) / 1e12,
                'note': 'time includes the slicing kernels of each split GETT'}

    def per_launch_roofline(fp64_peak, hbm_gbs):
        """gett_f64 launches against their own bound: max(FLOPs / DGEMM peak, algorithmic bytes / HBM)."""
        bound = spent = alg_bytes = 0.0
        nl = 0
        try:
            lines = open(dump).read().split('\n')
            os.remove(dump)
        except OSError:
            return None
        for ln in lines:
            f = ln.split()
            if len(f) < 13 or f[1] != 'GETT' or f[2] != '0':
                continue
            M, N, K, beta, ms, fl = int(f[4]), int(f[5]), int(f[6]), int(f[9]), float(f[10]), float(f[12])
            if M * N == 0 or ms <= 0:
                continue
            keff = fl / (2.0 * M * N)
            by = 8.0 * (M + N) * keff + (16.0 if beta else 8.0) * M * N
            bound += max(fl / (fp64_peak * 1e12), by / (hbm_gbs * 1e9)) * 1e3
            spent += ms
            nl += 1
            alg_bytes += by
        if not spent:
            return None
        return {'frac': bound / spent, 'bound_ms': bound / 2, 'spent_ms': spent / 2, 'launches': nl // 2,
                'algorithmic_bytes_per_launch': alg_bytes / nl,
                'note': 'per launch max(2MNK / measured DGEMM peak, 8(M+N)K + 8 or 16 MN bytes / measured HBM), '
                        'summed over the gett_f64 launches of 2 eager sweeps, over their summed event times'}

    if kname == 'assemble':
        # bytes: every gather term of every canonical element + the block written once (8 B each)
        roofline = {'bound': 'hbm', 'achieved': None, 'peak': peaks_file['hbm_gbs'], 'unit': 'GB/s', 'frac': None}
    else:
        roofline = dict(gett_line(kname))
    plb = per_launch_roofline(fp64_peak, peaks_file['hbm_gbs'])
    roofline.update({'kernel': kname, 'traffic': GETT_F64_TRAFFIC if kname == 'gett_f64' else None,
                     'shares': shares, 'per_sweep': per_sweep, 'per_launch_bound': plb,
                     'secondary': {k: gett_line(k) for k in ('gett_f64', 'gett_split') if k != kname},
                     'traffic_note': GETT_F64_TRAFFIC_NOTE + (
                         '; algorithmic bytes per launch of this run: %.1f MB' % (plb['algorithmic_bytes_per_launch'] / 1e6)
                         if plb else ''),
                     'note': 'achieved = algorithmic FLOPs of all launches of that kernel in 2 eager sweeps (CUDA '
                             'events around every launch) / their summed durations'})

    # end-to-end through the C ABI with host buffers: every step reads the t_vec from pinned host memory
    # and writes it back (ccq_b200_iterate_host: the T3 blocks are read at their canonical elements inside
    # the sweep, every block is copied out as soon as the sweep has written it)
    pinned = torch.empty(ctx.t_size, dtype=torch.float64, pin_memory=True)
    pinned.copy_(torch.from_numpy(ctx.get_t()))
    # warm-up over one DIIS cycle: captures the sweep graph with its copies and the DIIS iteration's graph
    for _ in range(6):
        ctx.iterate_host(it, pinned.data_ptr(), pinned.data_ptr())
        it += 1
    barrier(world)
    io_in = io_out = 0
    t0 = time.perf_counter()
    for k in range(args.steps):
        ctx.iterate_host(it, pinned.data_ptr(), pinned.data_ptr())
        h2d, d2h = ctx.io_bytes()
        io_in += h2d
        io_out += d2h + 16   # and the energy and residuum
        it += 1
    torch.cuda.synchronize()
    barrier(world)
    e2e_s = allmax(time.perf_counter() - t0, world) / (world * args.steps)
    ctx.close()

    # convergence to tol with the headline path, |dE| vs the FP64 oracle fixture
    conv = None
    if not args.no_converge:
        from ccq_b200 import config, driver
        c2 = new_ctx()
        cfg = config.Config(calc_type='CCSDT', tol=1e-10, diis_space=5, max_iter=100,
                            gpu_precision=headline, gpu_slices=args.slices,
                            gpu_autotune=not args.no_tune).calc_macros()
        r = driver.solve_cc(c2, cfg, out=lambda x: None)
        c2.close()
        g = golden_c2()
        conv = {'iterations': r.iterations, 'e_cor': r.e_cor, 'failed': r.failed,
                'dE_vs_fp64_oracle': (abs(r.e_cor - g['e_cor']) if g else None),
                'oracle': 'tests/golden/synthetic.json c2_ccsdt' if g else 'fixture missing',
                'split_iterations': sum(1 for h in r.history if h['split'])}

    batched = None if args.no_batch else batch_leg(rank, world)

    ccsdt_act = None
    if rank == 0 and not args.no_ccsdt:
        try:
            ccsdt_act = ccsdt_active_leg(s)
            ccsdt_act['ccsdt_fp64_s_per_iter'] = results['fp64']['s_per_iter']
            ccsdt_act['speedup_vs_ccsdt_fp64'] = results['fp64']['s_per_iter'] / ccsdt_act['s_per_iter']
            ccsdt_act['flops_fraction_of_ccsdt'] = ccsdt_act['flops_per_iter'] / results['fp64']['flops_per_iter']
        except Exception as ex:  # noqa: BLE001
            ccsdt_act = {'error': f'{type(ex).__name__}: {str(ex)[:200]}'}

    warm = None
    if rank == 0 and not args.no_warmstart:
        try:
            from ccq_b200 import warmstart
            warm = warmstart.study('CCSDT', 24, 10)
            warm.pop('loss_history', None)
        except Exception as ex:  # noqa: BLE001  (a failed extra leg must not cost the headline line)
            warm = {'error': f'{type(ex).__name__}: {str(ex)[:200]}'}

    crcc = None
    if rank == 0 and not args.no_crcc:
        try:
            crcc = crcc_leg(cpu_sample=(world == 1 and not args.no_cpu_baseline))
        except Exception as ex:  # noqa: BLE001
            crcc = {'error': f'{type(ex).__name__}: {str(ex)[:200]}'}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        r = cpu_reference(s, 1, 0, budget_s=60.0)
        cpu = {'value': r['s_per_iter'], 'unit': 's/iter', 'cores': r['cores'], 'kind': 'port',
               'sample': 'first CCSDT iteration of the same workload (one full update sweep + energy + ring); '
                         + BASELINE_KIND}
    if rank == 0:
        line = {
            'metric': METRIC, 'value': head['s_per_iter'], 'unit': 's/iter', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': head['s_per_iter'] * 1e3 * world,
            'higher_is_better': False, 'scaling': 'weak', 'vs_baseline': None,
            'dtype': 'f64' if headline == 'fp64' else f'f64 (int8 x{args.slices} slices, int32 acc)',
            'data': 'synthetic (seeded generator, no molecular integrals)',
            # the same workload config as the reference arm's line; how this arm ran it is in precision
            'config': {'workload': WORKLOAD, 'parallelism': f'replicas x{world}', 'l2': L2_NOTE},
            'precision': headline,
            'tflops': head['tflops'],
            'flops_per_iter': head['flops_per_iter'],
            'flops_reference_per_iter': REFERENCE_FLOPS_C2,
            'tflops_reference_count': REFERENCE_FLOPS_C2 / head['s_per_iter'] / 1e12,
            'flops_note': 'tflops = this engine\'s own GETT FLOPs per iteration / time; tflops_reference_count = the '
                          'reference algorithm\'s static FLOP count per iteration / the same time',
            'legs': results, 'autotune': tuning or None,
            'speedup_split_vs_fp64': (results['fp64']['s_per_iter'] / results['split']['s_per_iter']
                                      if 'split' in results else None),
            'roofline': roofline,
            'cpu_baseline': cpu,
            'e2e': {'value': e2e_s, 'unit': 's/iter', 'h2d_bytes_per_step': io_in // args.steps,
                    'd2h_bytes_per_step': io_out // args.steps,
                    'note': 'T1/T2 copied whole, T3 blocks read from the host at their canonical elements (the '
                            'rest are their antisymmetric images); every block copied back out as the sweep '
                            'finishes it, or the whole extrapolated vector after a DIIS step'},
            'gpu_launches': head['launches_per_iter'] * args.steps,
            'clocks': clk, 'convergence': conv, 'crcc23': crcc, 'batched_ccsd': batched, 'warm_start': warm,
            'ccsdt_active': ccsdt_act,
            'peaks': {'live': peaks_live, 'file': peaks_file, 'file_kind': peaks_kind},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
