"""ctypes binding of ``libccq_b200.so`` (the C ABI of ``include/ccq_b200.h``).

This is the same boundary a Fortran build of ccq binds with ISO_C_BINDING.
There is no CPU fallback: if the library is missing or no GPU is present the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libccq_b200.so')

PREC_FP64 = 0
PREC_SPLIT = 1

_lib = None

I64 = C.c_int64
DP = C.POINTER(C.c_double)


class CCQB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f'ccq_b200 error {code}: {msg}')
        self.code = code


class Dims(C.Structure):
    _fields_ = [('froz', I64), ('occ_a', I64), ('occ_b', I64), ('orbs', I64)]


class InitOpts(C.Structure):
    _fields_ = [('rowmajor', I64), ('act_occ_b', I64), ('act_unocc_a', I64)]


SIGNATURES = {
    'ccq_b200_egemm': (C.c_int, [I64, I64, I64, DP, DP, DP]),
    'ccq_b200_egemm_split': (C.c_int, [I64, I64, I64, DP, DP, DP, I64]),
    'ccq_b200_egemm_split_kernel': (C.c_int, [I64, I64, I64, DP, DP, DP, I64, I64]),
    'ccq_b200_egemm1': (C.c_int, [I64, I64, DP, DP, DP]),
    'ccq_b200_egemm2': (C.c_int, [I64, I64, DP, DP, DP]),
    'ccq_b200_init': (C.c_int, [C.POINTER(Dims), C.c_char_p, DP, DP, DP, DP, DP, I64, C.c_double, I64,
                                C.POINTER(C.c_void_p)]),
    'ccq_b200_init_rowmajor': (C.c_int, [C.POINTER(Dims), C.c_char_p, DP, DP, DP, DP, DP, I64, C.c_double, I64,
                                C.POINTER(C.c_void_p)]),
    'ccq_b200_init_ex': (C.c_int, [C.POINTER(Dims), C.c_char_p, C.c_void_p, DP, DP, DP, DP, DP, I64, C.c_double,
                                   I64, C.POINTER(C.c_void_p)]),
    'ccq_b200_t_size_act': (I64, [C.POINTER(Dims), I64, I64]),
    'ccq_b200_t_compress': (C.c_int, [C.POINTER(Dims), I64, I64, DP, I64, DP, I64]),
    'ccq_b200_t_expand': (C.c_int, [C.POINTER(Dims), I64, I64, DP, I64, DP, I64]),
    'ccq_b200_batch_create': (C.c_int, [C.POINTER(C.c_void_p), I64, C.POINTER(C.c_void_p)]),
    'ccq_b200_batch_iterate': (C.c_int, [C.c_void_p, I64, C.POINTER(I64), DP, DP, C.POINTER(I64)]),
    'ccq_b200_batch_stats': (C.c_int, [C.c_void_p, C.POINTER(I64), C.POINTER(C.c_double)]),
    'ccq_b200_batch_free': (C.c_int, [C.c_void_p]),
    'ccq_b200_sizes': (C.c_int, [C.c_void_p, C.POINTER(I64), C.POINTER(I64)]),
    'ccq_b200_set_t': (C.c_int, [C.c_void_p, DP, I64]),
    'ccq_b200_get_t': (C.c_int, [C.c_void_p, DP, I64]),
    'ccq_b200_block': (C.c_int, [C.c_void_p, C.c_char_p, DP, I64, I64]),
    'ccq_b200_update': (C.c_int, [C.c_void_p]),
    'ccq_b200_energy': (C.c_int, [C.c_void_p, DP]),
    'ccq_b200_iterate': (C.c_int, [C.c_void_p, I64, DP, DP, C.POINTER(I64)]),
    'ccq_b200_iterate_async': (C.c_int, [C.c_void_p, I64]),
    'ccq_b200_iterate_host': (C.c_int, [C.c_void_p, I64, C.c_void_p, C.c_void_p, I64, DP, DP, C.POINTER(I64)]),
    'ccq_b200_io_bytes': (C.c_int, [C.c_void_p, C.POINTER(I64), C.POINTER(I64)]),
    'ccq_b200_iterate_wait': (C.c_int, [C.c_void_p, DP, DP, C.POINTER(I64)]),
    'ccq_b200_lambda_init': (C.c_int, [C.c_void_p, C.c_double]),
    'ccq_b200_lambda_iterate': (C.c_int, [C.c_void_p, I64, DP, DP, C.POINTER(I64)]),
    'ccq_b200_crcc23': (C.c_int, [C.c_void_p, DP]),
    'ccq_b200_get_l': (C.c_int, [C.c_void_p, DP, I64]),
    'ccq_b200_set_precision': (C.c_int, [C.c_void_p, I64, I64]),
    'ccq_b200_autotune': (C.c_int, [C.c_void_p, I64, DP, DP]),
    'ccq_b200_force_tile': (C.c_int, [C.c_void_p, I64]),
    'ccq_b200_set_active': (C.c_int, [C.c_void_p, I64, I64]),
    'ccq_b200_set_external': (C.c_int, [C.c_void_p, I64]),
    'ccq_b200_use_graph': (C.c_int, [C.c_void_p, I64]),
    'ccq_b200_stats': (C.c_int, [C.c_void_p, C.POINTER(I64), DP, DP]),
    'ccq_b200_timing': (C.c_int, [C.c_void_p, DP, DP]),
    'ccq_b200_profile': (C.c_int, [C.c_void_p, I64]),
    'ccq_b200_profile_get': (C.c_int, [C.c_void_p, I64, DP, DP, C.POINTER(I64)]),
    'ccq_b200_free': (C.c_int, [C.c_void_p]),
    'ccq_b200_last_error': (C.c_int, [C.c_char_p, I64]),
    'ccq_b200_checkpoint_save': (C.c_int, [C.c_void_p, C.c_char_p, I64, I64, DP]),
    'ccq_b200_checkpoint_load': (C.c_int, [C.c_void_p, C.c_char_p, C.POINTER(I64), DP, C.POINTER(I64)]),
    'ccq_b200_checkpoint_info': (C.c_int, [C.c_char_p, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), DP,
                                           C.c_char_p, I64]),
    'ccq_b200_fcidump_header': (C.c_int, [C.c_char_p, C.POINTER(I64), C.POINTER(I64)]),
    'ccq_b200_fcidump_read': (C.c_int, [C.c_char_p, I64, DP, DP, DP]),
    'ccq_b200_fcidump_read_device': (C.c_int, [C.c_char_p, I64, DP, C.c_void_p, DP, C.c_void_p]),
    'ccq_b200_walkers_read': (C.c_int, [C.c_char_p, C.c_void_p, I64, I64, DP, I64, DP, I64, DP]),
}


def load(path=LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise CCQB200Error(-6, f'{path} not built (python -m ccq_b200.build)')
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _err(code):
    if code != 0:
        buf = C.create_string_buffer(1024)
        _lib.ccq_b200_last_error(buf, 1024)
        raise CCQB200Error(code, buf.value.decode(errors='replace'))


def _p(a):
    return a.ctypes.data_as(DP)


def fcidump_header(path):
    """(NORB, NELEC) of a FCIDUMP header (-1 for a key that is absent)."""
    lib = load()
    n, e = I64(), I64()
    _err(lib.ccq_b200_fcidump_header(os.fsencode(path), C.byref(n), C.byref(e)))
    return n.value, e.value


def fcidump_read(path, norb):
    """e1int[i, a], e2int[i, j, a, b] = <ij|ab> (index meaning of the reference's arrays), E_nuc."""
    lib = load()
    e1 = np.zeros((norb, norb), order='F')
    e2 = np.zeros((norb, norb, norb, norb), order='F')
    en = C.c_double()
    _err(lib.ccq_b200_fcidump_read(os.fsencode(path), norb, _p(e1), _p(e2), C.byref(en)))
    return np.ascontiguousarray(e1), np.ascontiguousarray(e2), en.value


def fcidump_read_device(path, norb, e2_dev_ptr, stream=0):
    """As fcidump_read, with e2int (Fortran order, norb^4 doubles) expanded into device memory."""
    lib = load()
    e1 = np.zeros((norb, norb), order='F')
    en = C.c_double()
    _err(lib.ccq_b200_fcidump_read_device(os.fsencode(path), norb, _p(e1), C.c_void_p(e2_dev_ptr), C.byref(en),
                                          C.c_void_p(stream)))
    return np.ascontiguousarray(e1), en.value


def walkers_read(path, froz, occ_a, occ_b, orbs, nel, with_sd=True, t4=True):
    """Cluster amplitudes of a FCIQMC walker file: (t_vec with T1..T3, {T4A..T4E: block} or None,
    dict(c_hf, records, quadruples, higher))."""
    from . import integrals as I
    lib = load()
    lay = I.TLayout(I.Dims(froz, occ_a, occ_b, orbs))
    t = np.zeros(lay.t_size)
    n4 = sum(int(np.prod(s)) for s in lay.t4_shape.values())
    t4v = np.zeros(n4) if t4 else None
    info = np.zeros(4)
    dims = Dims(froz, occ_a, occ_b, orbs)
    _err(lib.ccq_b200_walkers_read(os.fsencode(path), C.byref(dims), nel, int(bool(with_sd)), _p(t), t.size,
                                   _p(t4v) if t4 else None, n4 if t4 else 0, _p(info)))
    blocks = None
    if t4:
        blocks, off = {}, 0
        for b in I.T4_ORDER:
            shp = lay.t4_shape[b]
            k = int(np.prod(shp))
            blocks[b] = t4v[off:off + k].reshape(shp)
            off += k
    return t, blocks, dict(c_hf=info[0], records=int(info[1]), quadruples=int(info[2]), higher=int(info[3]))


def checkpoint_info(path):
    """Header of a checkpoint: dict(calc_type, dims, iteration, with_ring, state)."""
    lib = load()
    dims = (I64 * 9)()
    it, ring = I64(), I64()
    st = np.zeros(8)
    buf = C.create_string_buffer(32)
    _err(lib.ccq_b200_checkpoint_info(os.fsencode(path), dims, C.byref(it), C.byref(ring), _p(st), buf, 32))
    names = ('froz', 'oa', 'ob', 'va', 'vb', 'rhf', 'diis_space', 't_dev', 'vec_size')
    return dict(calc_type=buf.value.decode(), dims=dict(zip(names, list(dims))), iteration=it.value,
                with_ring=bool(ring.value), state=st)


def t_size_act(froz, occ_a, occ_b, orbs, act_occ_b, act_unocc_a):
    """Length of ccq's compressed CCSDt T vector (get_t_sizes_act)."""
    n = load().ccq_b200_t_size_act(C.byref(Dims(froz, occ_a, occ_b, orbs)), act_occ_b, act_unocc_a)
    if n < 0:
        _err(int(n))
    return int(n)


def t_compress(dims, act_occ_b, act_unocc_a, t_full):
    """Full-block T vector -> ccq's compressed CCSDt T vector (dims = (froz, occ_a, occ_b, orbs))."""
    d = Dims(*dims)
    t = np.ascontiguousarray(t_full, dtype=np.float64)
    out = np.empty(t_size_act(*dims, act_occ_b, act_unocc_a))
    _err(load().ccq_b200_t_compress(C.byref(d), act_occ_b, act_unocc_a, _p(t), t.size, _p(out), out.size))
    return out


def t_expand(dims, act_occ_b, act_unocc_a, t_act, n_full):
    """ccq's compressed CCSDt T vector -> full-block T vector of length n_full."""
    d = Dims(*dims)
    t = np.ascontiguousarray(t_act, dtype=np.float64)
    out = np.empty(n_full)
    _err(load().ccq_b200_t_expand(C.byref(d), act_occ_b, act_unocc_a, _p(t), t.size, _p(out), out.size))
    return out


def egemm(k1, k2, k3, A, B):
    """C(k2,k1) = B(k3,k2)^T A(k3,k1) on Fortran-ordered host arrays."""
    lib = load()
    A = np.asfortranarray(A, dtype=np.float64).reshape((k3, k1), order='F')
    B = np.asfortranarray(B, dtype=np.float64).reshape((k3, k2), order='F')
    Cm = np.zeros((k2, k1), order='F')
    _err(lib.ccq_b200_egemm(k1, k2, k3, _p(A), _p(B), _p(Cm)))
    return Cm


def egemm_split(k1, k2, k3, A, B, nslices=4, persistent=None):
    """egemm with int8 Ozaki slices on the tcgen05 tensor pipe (persistent: pick the kernel)."""
    lib = load()
    A = np.asfortranarray(A, dtype=np.float64).reshape((k3, k1), order='F')
    B = np.asfortranarray(B, dtype=np.float64).reshape((k3, k2), order='F')
    Cm = np.zeros((k2, k1), order='F')
    if persistent is None:
        _err(lib.ccq_b200_egemm_split(k1, k2, k3, _p(A), _p(B), _p(Cm), nslices))
    else:
        _err(lib.ccq_b200_egemm_split_kernel(k1, k2, k3, _p(A), _p(B), _p(Cm), nslices, int(persistent)))
    return Cm


def egemm1(k1, k3, A, B):
    lib = load()
    A = np.asfortranarray(A, dtype=np.float64).reshape((k3, k1), order='F')
    B = np.ascontiguousarray(B, dtype=np.float64).reshape(k3)
    Cv = np.zeros(k1)
    _err(lib.ccq_b200_egemm1(k1, k3, _p(A), _p(B), _p(Cv)))
    return Cv


def egemm2(k2, k3, A, B):
    lib = load()
    A = np.ascontiguousarray(A, dtype=np.float64).reshape(k3)
    B = np.asfortranarray(B, dtype=np.float64).reshape((k3, k2), order='F')
    Cv = np.zeros(k2)
    _err(lib.ccq_b200_egemm2(k2, k3, _p(A), _p(B), _p(Cv)))
    return Cv


class Batch:
    """Contexts of one plan iterated together (ccq_b200_batch_*): operation k of every active context
    runs as one launch."""

    def __init__(self, contexts):
        self._lib = load()
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.ptr.value for c in self.contexts])
        self.ptr = C.c_void_p()
        _err(self._lib.ccq_b200_batch_create(arr, len(self.contexts), C.byref(self.ptr)))

    def iterate(self, it, active):
        """One iteration of every context j with active[j]; returns (e_cor, residuum, did_diis) arrays."""
        n = len(self.contexts)
        act = np.ascontiguousarray(np.asarray(active, dtype=np.int64))
        e, r = np.zeros(n), np.zeros(n)
        d = np.zeros(n, dtype=np.int64)
        _err(self._lib.ccq_b200_batch_iterate(self.ptr, it, act.ctypes.data_as(C.POINTER(I64)), _p(e), _p(r),
                                              d.ctypes.data_as(C.POINTER(I64))))
        return e, r, d

    def stats(self):
        n, ms = I64(), C.c_double()
        _err(self._lib.ccq_b200_batch_stats(self.ptr, C.byref(n), C.byref(ms)))
        return {'launches': n.value, 'sweep_ms': ms.value}

    def close(self):
        if self.ptr:
            self._lib.ccq_b200_batch_free(self.ptr)
            self.ptr = C.c_void_p()


class Context:
    """A resident CC solve on the current CUDA device."""

    def __init__(self, froz, occ_a, occ_b, orbs, calc_type, f_a, f_b, v_aa, v_ab, v_bb,
                 rhf=False, shift=0.0, diis_space=5, active=None):
        """active = (act_occ_b, act_unocc_a) with calc_type 'CCSDt' (ccq_b200_init_ex)."""
        lib = load()
        self._lib = lib
        self.ptr = C.c_void_p()
        d = Dims(froz, occ_a, occ_b, orbs)
        arrs = (f_a, f_b, v_aa, v_ab, v_bb)
        if all(isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags.c_contiguous for x in arrs):
            # row-major arrays go in as they are (ccq_b200_init_rowmajor): no transposed copies
            self._keep = arrs
            init = lib.ccq_b200_init_rowmajor
        else:
            # Fortran (column-major) layout, as sys%ints arrays are in ccq
            self._keep = [np.asfortranarray(x, dtype=np.float64) for x in arrs]
            init = lib.ccq_b200_init
        fa, fb, vaa, vab, vbb = self._keep
        if active is not None or calc_type == 'CCSDt':
            m1, m2 = active if active is not None else (-1, -1)
            opts = InitOpts(int(init == lib.ccq_b200_init_rowmajor), int(m1), int(m2))
            _err(lib.ccq_b200_init_ex(C.byref(d), calc_type.encode(), C.cast(C.pointer(opts), C.c_void_p), _p(fa),
                                      _p(fb), _p(vaa), _p(vab), _p(vbb), int(bool(rhf)), float(shift),
                                      int(diis_space), C.byref(self.ptr)))
        else:
            _err(init(C.byref(d), calc_type.encode(), _p(fa), _p(fb), _p(vaa), _p(vab), _p(vbb),
                      int(bool(rhf)), float(shift), int(diis_space), C.byref(self.ptr)))
        self.dims = d
        self.active = active
        self._keep = None
        ts, vs = I64(), I64()
        _err(lib.ccq_b200_sizes(self.ptr, C.byref(ts), C.byref(vs)))
        self.t_size, self.vec_size = ts.value, vs.value

    def set_t(self, t):
        t = np.ascontiguousarray(t, dtype=np.float64)
        _err(self._lib.ccq_b200_set_t(self.ptr, _p(t), t.size))

    def get_t(self):
        t = np.empty(self.t_size)
        _err(self._lib.ccq_b200_get_t(self.ptr, _p(t), t.size))
        return t

    def get_block(self, name, shape):
        out = np.empty(shape)
        _err(self._lib.ccq_b200_block(self.ptr, name.encode(), _p(out), out.size, 0))
        return out

    def set_block(self, name, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        _err(self._lib.ccq_b200_block(self.ptr, name.encode(), _p(a), a.size, 1))

    def update(self):
        _err(self._lib.ccq_b200_update(self.ptr))

    def energy(self):
        e = C.c_double()
        _err(self._lib.ccq_b200_energy(self.ptr, C.byref(e)))
        return e.value

    def iterate(self, it):
        e, r, d = C.c_double(), C.c_double(), I64()
        _err(self._lib.ccq_b200_iterate(self.ptr, it, C.byref(e), C.byref(r), C.byref(d)))
        return e.value, r.value, bool(d.value)

    def io_bytes(self):
        """(host-to-device, device-to-host) bytes of the last iterate_host."""
        a, b = I64(), I64()
        _err(self._lib.ccq_b200_io_bytes(self.ptr, C.byref(a), C.byref(b)))
        return a.value, b.value

    def iterate_host(self, it, t_in_ptr, t_out_ptr):
        """One iteration from host t_vec t_in to host t_vec t_out (pointers to t_size doubles, pinned
        for overlap): block copies overlap the sweep.  Returns (e_cor, residuum, did_diis)."""
        e, r, d = C.c_double(), C.c_double(), I64()
        _err(self._lib.ccq_b200_iterate_host(self.ptr, it, C.c_void_p(t_in_ptr), C.c_void_p(t_out_ptr), self.t_size,
                                             C.byref(e), C.byref(r), C.byref(d)))
        return e.value, r.value, bool(d.value)

    def iterate_async(self, it):
        _err(self._lib.ccq_b200_iterate_async(self.ptr, it))

    def iterate_wait(self):
        e, r, d = C.c_double(), C.c_double(), I64()
        _err(self._lib.ccq_b200_iterate_wait(self.ptr, C.byref(e), C.byref(r), C.byref(d)))
        return e.value, r.value, bool(d.value)

    # -- CR-CC(2,3) (contexts created with calc_type 'CR-CC(2,3)') ---------------
    def lambda_init(self, e_cor):
        _err(self._lib.ccq_b200_lambda_init(self.ptr, float(e_cor)))

    def lambda_iterate(self, it):
        e, r, d = C.c_double(), C.c_double(), I64()
        _err(self._lib.ccq_b200_lambda_iterate(self.ptr, it, C.byref(e), C.byref(r), C.byref(d)))
        return e.value, r.value, bool(d.value)

    def crcc23(self):
        e = np.zeros(4)
        _err(self._lib.ccq_b200_crcc23(self.ptr, _p(e)))
        return e

    def get_l(self):
        out = np.empty(self.vec_size)
        _err(self._lib.ccq_b200_get_l(self.ptr, _p(out), out.size))
        return out

    def autotune(self, reps=3):
        """Times every contraction's candidate configurations once; returns (ms before, ms after)."""
        a, b = C.c_double(), C.c_double()
        _err(self._lib.ccq_b200_autotune(self.ptr, reps, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_external(self, on=True):
        """Externally corrected CC: T3 / T4 held at their set values, only T1 and T2 iterate."""
        _err(self._lib.ccq_b200_set_external(self.ptr, int(bool(on))))

    def set_active(self, act_occ_b, act_unocc_a):
        """CCSDt: triples with >= 1 active occupied and >= 1 active virtual index (ccq's boundaries)."""
        _err(self._lib.ccq_b200_set_active(self.ptr, act_occ_b, act_unocc_a))

    def force_tile(self, tile):
        """Every contraction on one kernel family (0 shape default, 1 64x64, 2 skinny, 3 small-K, 4 64x64 3-stage,
        5 skinny 2-stage, 6 register-direct small-K)."""
        _err(self._lib.ccq_b200_force_tile(self.ptr, tile))

    def save_checkpoint(self, path, iteration=0, state=None, with_ring=True):
        """Resident t_vec, T4 blocks and (with_ring) the DIIS ring to ``path``."""
        st = np.zeros(8)
        if state is not None:
            st[:len(state)] = state
        _err(self._lib.ccq_b200_checkpoint_save(self.ptr, os.fsencode(path), int(with_ring), iteration, _p(st)))

    def load_checkpoint(self, path):
        """Restores a checkpoint; returns (iteration, state[8], with_ring)."""
        it, ring = I64(), I64()
        st = np.zeros(8)
        _err(self._lib.ccq_b200_checkpoint_load(self.ptr, os.fsencode(path), C.byref(it), _p(st), C.byref(ring)))
        return it.value, st, bool(ring.value)

    def set_precision(self, mode, nslices=4):
        _err(self._lib.ccq_b200_set_precision(self.ptr, mode, nslices))

    def use_graph(self, enable=True):
        """True / 1: concurrent graph, 2: single-stream graph, False / 0: eager launches."""
        _err(self._lib.ccq_b200_use_graph(self.ptr, int(enable)))

    def stats(self):
        n, f, ms = I64(), C.c_double(), C.c_double()
        _err(self._lib.ccq_b200_stats(self.ptr, C.byref(n), C.byref(f), C.byref(ms)))
        return {'launches': n.value, 'flops': f.value, 'sweep_ms': ms.value}

    def timing(self):
        a, b = C.c_double(), C.c_double()
        _err(self._lib.ccq_b200_timing(self.ptr, C.byref(a), C.byref(b)))
        return a.value, b.value

    def profile(self, enable=True):
        _err(self._lib.ccq_b200_profile(self.ptr, int(bool(enable))))

    def profile_get(self):
        out = {}
        for k, name in enumerate(('gett_f64', 'gett_split', 'assemble', 'other')):
            ms, fl, n = C.c_double(), C.c_double(), I64()
            _err(self._lib.ccq_b200_profile_get(self.ptr, k, C.byref(ms), C.byref(fl), C.byref(n)))
            out[name] = {'ms': ms.value, 'flops': fl.value, 'launches': n.value}
        return out

    def set_t_ptr(self, ptr, n):
        """set_t from a raw host pointer (pinned buffers)."""
        _err(self._lib.ccq_b200_set_t(self.ptr, C.cast(ptr, DP), n))

    def get_t_ptr(self, ptr, n):
        _err(self._lib.ccq_b200_get_t(self.ptr, C.cast(ptr, DP), n))

    def close(self):
        if self.ptr:
            self._lib.ccq_b200_free(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def header_symbols(header=None):
    """Function names declared in include/ccq_b200.h."""
    import re
    header = header or os.path.join(HERE, '..', 'include', 'ccq_b200.h')
    text = open(header).read()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'^\s*(?:int|int64_t|void)\s+(\w+)\s*\(', text, flags=re.M)))
