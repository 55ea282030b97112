"""ccq-compatible driver on the resident GPU solver.

Keeps the reference's outer program and replaces only the amplitude update
underneath it:
  * ``run``            <- ``run_calcs``/``init_system`` (``src/calc_driver.f90:11-141``)
  * ``solve_cc``       <- ``solve_cc`` + ``jacobi_iter`` (``src/solve_cc.f90:12-269``):
    update, energy, ring write, residuum and DIIS every ``diis_space+1``
    iterations (inside ``Context.iterate``), the iteration table, the
    ``cc.comm`` stop file, NaN and max-iteration exits, and convergence when
    the last three |dE| are below tol (``:293-316``)
  * printing           <- ``print_iter_head``/``print_iteration``/``print_summary``
    (``src/printing.F90:260-349``)

Usage: ``python -m ccq_b200.driver input.inp``.
"""
from __future__ import annotations

import math
import os
import sys
import time

import numpy as np

from . import config as cfgmod
from . import integrals as I
from . import lib


class Result:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def print_iter_head(out):
    out(f"\n  {'It.':>4}{'E (Corr)':>15}{'dE':>15}{'Residuum':>15}{'Wall Time':>16}")
    out('  ' + '-' * 65)


def print_iteration(out, it, ecor, de, res, secs):
    nmin = int(secs) // 60
    nsec = secs - nmin * 60.0
    out(f'  {it:4d}{ecor:15.10f}{de:15.10f}{res:15.10f}{nmin:5d} min{nsec:5.1f} s')


def solve_cc(ctx, cfg, out=print, precision=None):
    """jacobi_iter on the device.  Returns a Result with energies and timings."""
    prec = precision or cfg.gpu_precision
    split = prec == 'split'
    ctx.set_precision(lib.PREC_SPLIT if split else lib.PREC_FP64, cfg.gpu_slices)
    ctx.use_graph(cfg.gpu_graph)
    if cfg.gpu_autotune:
        ctx.autotune()
    conv = [1.0, 1.0, 1.0]
    en_cor = 0.0
    failed = False
    hist = []
    it0 = 0
    fp64_iters = 0
    if cfg.restart:
        # continue from the checkpoint (src/solve_cc.f90:56-60 prints the restart energy; its
        # T1-T3 restart starts from zero, here the saved amplitudes and DIIS ring are resumed)
        path = cfg.bin_path()
        if not os.path.exists(path):
            raise ValueError('CONFIGURATION ERROR: Restart file not found')
        it_saved, state, with_ring = ctx.load_checkpoint(path)
        out(f"  {'Restart correlation energy':>27}  {ctx.energy():16.10f}\n")
        if with_ring:
            # the ring is resumed too: iteration numbering, DIIS schedule and convergence history go on
            it0 = it_saved
            en_cor, conv, fp64_iters = state[0], list(state[1:4]), int(state[4])
            if split and not state[5]:
                split = False
                ctx.set_precision(lib.PREC_FP64, cfg.gpu_slices)
    prev = time.time()
    print_iter_head(out)
    it = it0
    for it in range(it0 + 1, cfg.max_iter + 1):
        e_new, res, did = ctx.iterate(it)
        st = ctx.stats()
        diff = en_cor - e_new
        conv = [conv[1], conv[2], diff]
        en_cor = e_new
        if did:
            out('      DIIS cycle')
        now = time.time()
        print_iteration(out, it, e_new, diff, res, now - prev)
        hist.append(dict(e=e_new, de=diff, res=res, ms=st['sweep_ms'], split=split, launches=st['launches']))
        prev = now
        if not split:
            fp64_iters += 1
        if os.path.exists('cc.comm'):
            os.remove('cc.comm')
            out('Signaled to end')
            break
        if split and abs(diff) < cfg.gpu_fp64_finish:
            # hand over to FP64: the remaining iterations converge the exact equations
            split = False
            ctx.set_precision(lib.PREC_FP64, cfg.gpu_slices)
            out('      FP64 finish')
        if cfg.gpu_checkpoint_every and it % cfg.gpu_checkpoint_every == 0:
            ctx.save_checkpoint(cfg.bin_path(), it, solver_state(en_cor, conv, fp64_iters, split))
        if not split and fp64_iters >= 3 and all(abs(c) < cfg.tol for c in conv):
            break
        if math.isnan(e_new):
            out('FAILED TO CONVERGE')
            failed = True
            break
        if it == cfg.max_iter:
            out(f'FAILED TO CONVERGE IN {cfg.max_iter} ITERATIONS. KEEPING LAST T VECTOR.')
            failed = True
    return Result(e_cor=en_cor, iterations=it, failed=failed, history=hist,
                  state=solver_state(en_cor, conv, fp64_iters, split))


def solver_state(en_cor, conv, fp64_iters, split):
    """The host half of a checkpoint: energy, last three dE, FP64 iterations, split flag."""
    return [en_cor, conv[0], conv[1], conv[2], float(fp64_iters), float(split)]


def solve_lcc(ctx, cfg, e_cor, out=print):
    """solve_lcc (``src/solve_cc.f90:101-173``): jacobi_iter on lambda with the
    left energy sqrt(sum LH^2) + E_cor and the same convergence rule."""
    ctx.lambda_init(e_cor)
    out('Left Coupled cluster')
    out('--------------------')
    conv = [1.0, 1.0, 1.0]
    en = 0.0
    failed = False
    hist = []
    prev = time.time()
    print_iter_head(out)
    it = 0
    for it in range(1, cfg.max_iter + 1):
        e_new, res, did = ctx.lambda_iterate(it)
        diff = en - e_new
        conv = [conv[1], conv[2], diff]
        en = e_new
        if did:
            out('      DIIS cycle')
        now = time.time()
        print_iteration(out, it, e_new, diff, res, now - prev)
        hist.append(dict(e=e_new, de=diff, res=res))
        prev = now
        if all(abs(c) < cfg.tol for c in conv):
            break
        if math.isnan(e_new):
            out('FAILED TO CONVERGE')
            failed = True
            break
        if it == cfg.max_iter:
            out(f'FAILED TO CONVERGE IN {cfg.max_iter} ITERATIONS. KEEPING LAST T VECTOR.')
            failed = True
    return Result(e_left=en, iterations=it, failed=failed, history=hist)


def print_cct3(out, e_ref, e_cor, e23):
    """print_cct3 (``src/printing.F90:234-258``)."""
    out(f"\n{'Method':>20}{'Correlation (Eh)':>18}{'Total Energy (Eh)':>18}")
    out(' ' * 10 + '-' * 46)
    out(f"{'CCSDt':>20}{e_cor:18.12f}{e_ref + e_cor:18.12f}")
    for lab, x in zip(('CC(t;3),A', 'CC(t;3),B', 'CC(t;3),C', 'CC(t;3)'), e23):
        out(f'{lab:>20}{e_cor + x:18.12f}{e_ref + e_cor + x:18.12f}')


def load_system(cfg, base_dir='.'):
    def path(p):
        return p if os.path.isabs(p) else os.path.join(base_dir, p)
    if cfg.fcidump:
        e1, e2, enuc = I.read_fcidump(path(cfg.fcidump), cfg.orbs)
    else:
        e1 = I.read_onebody(path(cfg.onebody), cfg.orbs)
        e2, enuc = I.read_twobody(path(cfg.twobody), cfg.orbs)
    fa, fb = I.fock(e1, e2, cfg.occ_a, cfg.occ_b)
    vaa, vab, vbb = I.spin_blocks(e2, cfg.froz)
    eref = I.hf_energy(e1, e2, cfg.occ_a, cfg.occ_b) + enuc
    return dict(f_a=fa, f_b=fb, v_aa=vaa, v_ab=vab, v_bb=vbb, e_ref=eref)


def load_external(ctx, cfg, path, out=print):
    """Externally corrected CC: T3 (and for CCSDTQ T4) blocks from a .npz file (keys T3A..T3D, T4A..T4E,
    optionally T1A..T2C as the starting T1, T2), held fixed while T1 and T2 iterate
    (the role of ext_cor_driver's amplitudes, ``src/ext_cor/ext_cor.f90:12-149``)."""
    if cfg.calc_type not in ('CCSDT', 'CCSDTQ'):
        raise ValueError('CONFIGURATION ERROR: external amplitudes need calc_type CCSDT or CCSDTQ')
    if not os.path.exists(path):
        raise ValueError('CONFIGURATION ERROR: external amplitude file not found')
    z = np.load(path)
    lay = I.TLayout(I.Dims(cfg.froz, cfg.occ_a, cfg.occ_b, cfg.orbs))
    t = np.zeros(lay.t_size)
    for b in I.T_VEC_ORDER:
        if b in z.files:
            lay.view(t, b)[...] = z[b]
    ctx.set_t(t)
    if cfg.calc_type == 'CCSDTQ':
        for b, shp in lay.t4_shape.items():
            if b in z.files:
                ctx.set_block(b, np.asarray(z[b]).reshape(shp))
    ctx.set_external(True)
    out('  External T3' + (' and T4' if cfg.calc_type == 'CCSDTQ' else '') + ' amplitudes from ' + path)


def load_walkers(ctx, cfg, path, out=print):
    """CAD-FCIQMC (external_correction_driver, ``src/ext_cor/ext_cor.f90:12-144``): the cluster analysis
    of the walker file gives T3 and T4, held fixed while T1 and T2 iterate from the analysed T1, T2
    (from zero with ext_cor_sd=.false.)."""
    out('Cluster analysis')
    out('----------------')
    t, t4, info = lib.walkers_read(path, cfg.froz, cfg.occ_a, cfg.occ_b, cfg.orbs, cfg.occ_a + cfg.occ_b,
                                   with_sd=cfg.ext_cor_sd)
    out(f"  {info['records']} determinants read from {path}; {info['quadruples']} quadruples, "
        f"{info['higher']} higher excitations skipped; Hartree-Fock coefficient {info['c_hf']:.10g}")
    ctx.set_t(t)
    for b, blk in t4.items():
        ctx.set_block(b, blk)
    ctx.set_external(True)
    out(f"\n  {'External correlation energy':>27}  {ctx.energy():16.10f}\n")


def run(input_path, out=print, base_dir='.'):
    cfg = cfgmod.parse(input_path)
    if cfg.fcidump:
        fp = cfg.fcidump if os.path.isabs(cfg.fcidump) else os.path.join(base_dir, cfg.fcidump)
        if not os.path.exists(fp):
            raise ValueError('CONFIGURATION ERROR: FCIDUMP file not found')
        cfgmod.apply_fcidump(cfg, fp)
    cfg.calc_macros()
    if not cfg.acc_default():
        bad = ', '.join(f'{k}={v}' for k, v in cfg.acc.items() if any(x != 1.0 for x in v))
        raise ValueError(f'CONFIGURATION ERROR: ACC diagram factors other than 1.0 are not served by this '
                         f'engine ({bad}); CCSD, CCSDT, CCSDTQ and their variants run with all factors 1.0')
    if cfg.output_log:
        # output_log (src/parser.f90:719-720): the calculation's output also goes to that file
        path = cfg.output_log if os.path.isabs(cfg.output_log) else os.path.join(base_dir, cfg.output_log)
        log = open(path, 'w')
        out0 = out

        def out(line, _log=log, _out=out0):
            _out(line)
            _log.write(line + '\n')
            _log.flush()
    if cfg.echo:
        # print_config / echo: the input file as read
        out('Input configuration')
        for ln in cfg.lines:
            out('  ' + ln)
    sysd = load_system(cfg, base_dir)
    out('Calculation parameters: ' + cfgmod.format_config(cfg))
    out(f"  Reference energy {sysd['e_ref']:.12f}")
    out('Coupled cluster')
    out('---------------')
    # CCSDt (and the CCSDt part of CC(t;3)): the CCSDT plan restricted to the active triples
    active = cfg.calc_type in ('CCSDt', 'CC(t;3)')

    def context(ctype):
        act = (cfg.act_occ_b, cfg.act_unocc_a) if ctype == 'CCSDt' else None
        return lib.Context(cfg.froz, cfg.occ_a, cfg.occ_b, cfg.orbs, ctype, sysd['f_a'], sysd['f_b'],
                           sysd['v_aa'], sysd['v_ab'], sysd['v_bb'], rhf=cfg.rhf, shift=cfg.shift,
                           diis_space=cfg.diis_space, active=act)
    walkers = None
    if cfg.calc_type == 'CADFCIQMC':
        if cfg.ext_cor_file_h5:
            raise ValueError('CONFIGURATION ERROR: HDF5 walker files (ext_cor_file_h5) need an HDF5 library, '
                             'which this build does not have')
        walkers = cfg.ext_cor_file if os.path.isabs(cfg.ext_cor_file) else os.path.join(base_dir, cfg.ext_cor_file)
        if not cfg.ext_cor_file or not os.path.exists(walkers):
            raise ValueError('CONFIGURATION ERROR: Walkers file not found')
    ctx = context('CCSDt' if active else 'CCSDTQ' if walkers else cfg.calc_type)
    if walkers:
        load_walkers(ctx, cfg, walkers, out)
    if cfg.gpu_external_t:
        load_external(ctx, cfg, cfg.gpu_external_t if os.path.isabs(cfg.gpu_external_t)
                      else os.path.join(base_dir, cfg.gpu_external_t), out)
    cfg.bin_file = cfg.bin_path()
    if not os.path.isabs(cfg.bin_file):
        cfg.bin_file = os.path.join(base_dir, cfg.bin_file)
    try:
        r = solve_cc(ctx, cfg, out)
        if cfg.keep_bin:
            # final amplitudes and ring: restart= continues an unconverged run exactly
            ctx.save_checkpoint(cfg.bin_path(), r.iterations, r.state)
        if cfg.calc_type == 'CR-CC(2,3)':
            # hbar2 + solve_lcc + crcc23 (src/calc_driver.f90:55-73)
            r.left = solve_lcc(ctx, cfg, r.e_cor, out)
            r.e23 = ctx.crcc23()
            print_cct3(out, sysd['e_ref'], r.e_cor, r.e23)
            r.e_ccsd = r.e_cor
            r.e_cor = r.e_cor + r.e23[3]
            r.failed = r.failed or r.left.failed
        elif cfg.calc_type == 'CC(t;3)':
            # hbar2 + solve_lcc + crcc23 (src/calc_driver.f90:55-73) on the CCSDt T1 and T2
            # (hbar2 reads t_vec(1:pos(6)-1), src/hbar.f90:71-73), the sums over the triples
            # outside the active space
            t = ctx.get_t()
            ctx.close()
            ctx = context('CR-CC(2,3)')
            ctx.set_active(cfg.act_occ_b, cfg.act_unocc_a)
            ctx.set_t(t[:ctx.t_size])
            r.left = solve_lcc(ctx, cfg, r.e_cor, out)
            r.e23 = ctx.crcc23()
            print_cct3(out, sysd['e_ref'], r.e_cor, r.e23)
            r.e_ccsdt = r.e_cor
            r.e_cor = r.e_cor + r.e23[3]
            r.failed = r.failed or r.left.failed
    finally:
        ctx.close()
    out('\nCalculation Summary (Eh)')
    out('------------------------')
    out(f"{'Reference':>20}{sysd['e_ref']:18.12f}")
    out(f"{'Correlation':>20}{r.e_cor:18.12f}")
    out(f"{cfg.calc_type:>20}{sysd['e_ref'] + r.e_cor:18.12f}")
    r.e_ref = sysd['e_ref']
    r.e_total = sysd['e_ref'] + r.e_cor
    return r


if __name__ == '__main__':
    res = run(sys.argv[1])
    sys.exit(1 if res.failed else 0)
