"""ccq input-file parser (keys and calc_type macros of ``src/parser.f90``).

  * ``parse``          <- ``get_config`` (``src/parser.f90:99-185``): a line
    containing ``#`` or ``!`` anywhere is skipped; ``key=value`` or bare flag keys
  * key aliases        <- ``get_sys_data`` (``:440-470``), ``get_run_opts``
    (``:638-732``), defaults of ``set_default_options`` (``:779-844``)
  * ``process``        <- ``process_sys_data`` (``:476-504``)
  * ``calc_macros``    <- ``get_calc_macros`` (``:316-432``)

New keys of this engine are prefixed ``gpu_``: ``gpu_precision`` (fp64 |
split), ``gpu_slices`` (int8 slices per operand), ``gpu_fp64_finish`` (|dE|
below which the split mode hands over to FP64), ``gpu_graph`` (replay each
sweep as one CUDA graph), ``gpu_autotune`` (time every contraction's tile and
split-K candidates once before the first iteration and keep the fastest),
``gpu_checkpoint_every`` (write the checkpoint every N iterations),
``gpu_external_t`` (externally corrected CC: T3 / T4 from a .npz file, held
fixed while T1 and T2 iterate).  The
reference's ``fcidump``, ``restart`` and ``output_bin`` keys are served:
``restart`` resumes t_vec, T4 and the DIIS ring from ``output_bin``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field


# get_acc_opts (src/parser.f90:527-542): key -> number of factors
ACC_KEYS = {'t2t2_t2': 5, 't3_t2': 2, 't1t3_t2': 4, 't2t2_t3': 3, 't2t3_t3': 5}


def _reals(val, n, key):
    """List-directed read of n reals (Fortran ``read(val, *) array``): blanks or commas separate."""
    toks = [t for t in val.replace(',', ' ').split() if t]
    if len(toks) < n:
        raise ValueError(f'CONFIGURATION ERROR: {key} needs {n} real values')
    try:
        return [float(t.replace('d', 'e').replace('D', 'E')) for t in toks[:n]]
    except ValueError:
        raise ValueError(f'CONFIGURATION ERROR: {key} must be {n} reals') from None


def _logical(val):
    v = val.strip().lower().strip('.')
    if v in ('true', 't', 'yes', '1'):
        return True
    if v in ('false', 'f', 'no', '0'):
        return False
    raise ValueError(f'CONFIGURATION ERROR: {val!r} must be logical')


def _ftrunc_div(a, b):
    return int(a / b) if b else 0


@dataclass
class Config:
    froz_spin: int = 0
    nel: int = -1
    nvirt: int = -1
    mult: int = 0
    rhf: bool = False
    shift: float = 0.0
    max_iter: int = 60
    diis_space: int = 5
    tol: float = 1.0e-4
    calc_type: str = ''
    onebody: str = 'onebody.inp'
    twobody: str = 'twobody.inp'
    fcidump: str = ''
    bin_file: str = ''
    gpu_checkpoint_every: int = 0
    keep_bin: bool = True
    num_threads: int = 1
    restart: bool = False
    label: str = ''
    sym_file: str = ''
    gpu_precision: str = 'fp64'
    gpu_slices: int = 4
    gpu_fp64_finish: float = 1.0e-6
    gpu_graph: bool = True
    gpu_autotune: bool = False
    gpu_external_t: str = ''
    act_occ: int = -1
    act_unocc: int = -1
    ext_cor_file: str = ''
    ext_cor_sd: bool = True
    ext_cor_file_h5: bool = False
    # ACC diagram factors (acc_t, src/cc_types.f90:12-20), all 1.0 by default (src/parser.f90:838-842)
    acc: dict = field(default_factory=lambda: {k: [1.0] * n for k, n in ACC_KEYS.items()})
    # keys that get_calc_macros overwrites for every served calc_type (src/parser.f90:339-432)
    lvl_t_key: bool = False
    lvl_q_key: bool = False
    act_ind_t: int = 0
    act_ind_q: int = 0
    sorted_ints: bool = False
    echo: bool = False
    output_log: str = ''
    lines: list = field(default_factory=list)
    # derived (process_sys_data)
    froz: int = 0
    occ_a: int = 0
    occ_b: int = 0
    orbs: int = 0
    act_occ_b: int = 0
    act_unocc_a: int = 0
    lvl_t: bool = False
    lvl_q: bool = False
    extra: dict = field(default_factory=dict)

    def process(self):
        self.froz = self.froz_spin // 2
        self.occ_a = self.nel // 2
        self.occ_b = self.occ_a - _ftrunc_div(self.mult - 1, 2)
        self.orbs = (self.nel + self.nvirt) // 2
        # active space (process_sys_data, src/parser.f90:495-499)
        self.act_occ_b = max(self.occ_b - self.act_occ, self.froz)
        self.act_unocc_a = min(self.occ_a + self.act_unocc, self.orbs)
        return self

    def acc_default(self):
        """True when every ACC factor is 1.0 (the CC methods as derived)."""
        return all(x == 1.0 for v in self.acc.values() for x in v)

    def bin_path(self):
        """Checkpoint file: output_bin, else tvec_<label>.bin (tvec.bin without a label)."""
        if self.bin_file:
            return self.bin_file
        return f'tvec_{self.label}.bin' if self.label else 'tvec.bin'

    def calc_macros(self):
        if self.calc_type in ('CCT3', 'CCt3'):
            self.calc_type = 'CC(t;3)'    # src/parser.f90:400-401
        ct = self.calc_type
        if ct == 'CCSD':
            self.lvl_t, self.lvl_q = False, False
        elif ct == 'CCSDT':
            self.lvl_t, self.lvl_q = True, False
        elif ct == 'CCSDTQ':
            self.lvl_t, self.lvl_q = True, True
        elif ct == 'CCSDt':
            # src/parser.f90:380-388: active-space triples with act_ind_t = 1
            if self.act_occ == -1 and self.act_unocc == -1:
                raise ValueError('CONFIGURATION ERROR: Active space methods require an active space')
            self.lvl_t, self.lvl_q = True, False
        elif ct == 'CC(t;3)':
            # src/parser.f90:400-411: CCSDt, then hbar, left CCSD and the MM(2,3) correction over the
            # triples outside the active space.  ccq checks the active space only for CCSDt
            # (parser.f90:251-254); without one its act_occ_b = occ_b + 1 and act_unocc_a = occ_a - 1
            # lie outside the ranges its sorted integrals are built for, so it is required here too.
            if self.act_occ == -1 and self.act_unocc == -1:
                raise ValueError('CONFIGURATION ERROR: Active space methods require an active space')
            self.lvl_t, self.lvl_q = True, False
        elif ct == 'CADFCIQMC':
            # src/parser.f90:341-347: CCSD-level iterations with T3 and T4 from the walker file
            self.lvl_t, self.lvl_q = False, False
        elif ct == 'CR-CC(2,3)':
            # src/parser.f90:368-377: CCSD, then hbar, left CCSD and the MM(2,3) correction
            self.lvl_t, self.lvl_q = False, False
        elif ct == 'DCSD-MC':
            # src/parser.f90:350-358: CADFCIQMC-type external correction with the T2^2 diagrams of the
            # doubles scaled by (1, 0, 1/2, 1/2, 0), the dropped fractions taken from the walker T2
            self.acc['t2t2_t2'] = [1.0, 0.0, 0.5, 0.5, 0.0]
            self.lvl_t, self.lvl_q = False, False
        else:
            raise ValueError(f'calc_type {ct!r} is not served by this engine '
                             '(CCSD, CCSDT, CCSDTQ, CCSDt, CC(t;3), CR-CC(2,3), CADFCIQMC are; the others stay on the CPU program)')
        return self


def parse_lines(lines):
    cfg = Config()
    cfg.lines = [ln.rstrip('\n') for ln in lines]
    for raw in lines:
        line = raw.rstrip('\n')
        if '#' in line or '!' in line:
            continue
        if line.strip() == '':
            continue
        if '=' in line:
            k, v = line.split('=', 1)
            key, val = k.strip(), v.strip()
        else:
            key, val = line.strip(), ''
        _apply(cfg, key, val)
    return cfg.process()


def parse(path):
    with open(path) as fh:
        return parse_lines(fh.readlines())


def _apply(cfg, key, val):
    if key in ('core', 'nfroz', 'frozen', 'froz'):
        cfg.froz_spin = int(val)
    elif key in ('nel', 'electrons'):
        cfg.nel = int(val)
    elif key in ('nvir', 'nvirt', 'virtuals'):
        cfg.nvirt = int(val)
    elif key in ('multiplicity', 'mult'):
        cfg.mult = int(val)
    elif key == 'rhf':
        cfg.rhf = _logical(val)
    elif key == 'shift':
        cfg.shift = float(val.replace('d', 'e').replace('D', 'E'))
    elif key in ('max_iterations', 'max_iter'):
        cfg.max_iter = int(val)
    elif key in ('diis_space', 'diis'):
        cfg.diis_space = int(val)
    elif key in ('tolerance', 'tol', 'itol'):
        try:
            itol = int(val)
            cfg.tol = 10.0 ** itol
        except ValueError:
            cfg.tol = float(val.replace('d', 'e').replace('D', 'E'))
    elif key == 'calc_type':
        cfg.calc_type = val
    elif key in ('restart', 'rest'):
        cfg.restart = True
    elif key == 'label':
        cfg.label = val
    elif key == 'ext_cor_file':
        cfg.ext_cor_file = val
    elif key == 'ext_cor_sd':
        cfg.ext_cor_sd = _logical(val)
    elif key == 'ext_cor_file_h5':
        cfg.ext_cor_file_h5 = True
    elif key in ('symfile', 'sym_file'):
        cfg.sym_file = val
    elif key == 'onebody':
        cfg.onebody = val
    elif key == 'twobody':
        cfg.twobody = val
    elif key == 'fcidump':
        cfg.fcidump = val
    elif key == 'keep_bin':
        cfg.keep_bin = _logical(val)
    elif key == 'output_bin':
        cfg.bin_file = val
    elif key == 'gpu_checkpoint_every':
        cfg.gpu_checkpoint_every = int(val)
    elif key == 'num_threads':
        cfg.num_threads = int(val)
    elif key == 'gpu_precision':
        if val not in ('fp64', 'split'):
            raise ValueError('gpu_precision must be fp64 or split')
        cfg.gpu_precision = val
    elif key == 'gpu_slices':
        cfg.gpu_slices = int(val)
    elif key == 'gpu_fp64_finish':
        cfg.gpu_fp64_finish = float(val)
    elif key == 'gpu_graph':
        cfg.gpu_graph = _logical(val)
    elif key == 'gpu_autotune':
        cfg.gpu_autotune = _logical(val)
    elif key == 'gpu_external_t':
        cfg.gpu_external_t = val
    elif key == 'act_occ':
        cfg.act_occ = int(val)
    elif key == 'act_unocc':
        cfg.act_unocc = int(val)
    elif key in ACC_KEYS:
        cfg.acc[key] = _reals(val, ACC_KEYS[key], key)
    elif key in ('lvl_t', 'lvl_q'):
        # read, checked, then overwritten by get_calc_macros for every served calc_type
        try:
            setattr(cfg, key + '_key', _logical(val))
        except ValueError:
            raise ValueError(f'CONFIGURATION ERROR: {key} must logical') from None
    elif key in ('act_ind_t', 'act_ind_q'):
        setattr(cfg, key, int(val))
    elif key == 'sorted_ints':
        # ccq's sorted-integral code path for CCSDt; the integrals here are always resident in full
        cfg.sorted_ints = _logical(val)
    elif key in ('print_config', 'echo'):
        cfg.echo = True
    elif key == 'output_log':
        cfg.output_log = val
    elif key == 'ext_cor':
        # honoured by ccq only for calc_type=dev (src/parser.f90:619-623)
        cfg.extra[key] = val
    else:
        cfg.extra[key] = val


def apply_fcidump(cfg, path):
    """FCIDUMP override (``src/parser.f90:168-169``, ``get_fcidump`` ``:260-313``):
    nel = NELEC, nvirt = 2 NORB - NELEC, then the derived sizes again."""
    from . import lib
    norb, nelec = lib.fcidump_header(path)
    cfg.nel = nelec
    cfg.nvirt = 2 * norb - nelec
    return cfg.process()


def format_config(cfg):
    return (f'froz={cfg.froz} occ_a={cfg.occ_a} occ_b={cfg.occ_b} orbs={cfg.orbs} calc_type={cfg.calc_type} '
            f'tol={cfg.tol:.1e} diis_space={cfg.diis_space} shift={cfg.shift}')


def isclose(a, b):
    return math.isclose(a, b, rel_tol=0, abs_tol=1e-15)
