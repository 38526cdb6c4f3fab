"""ctypes binding of the engine C ABI (include/t3ns_b200.h).

Only plain pointers cross the boundary.  Device buffers are passed as raw
addresses (``torch.Tensor.data_ptr()`` or any other CUDA allocation).  There is
no CPU fallback: if the library is missing or a call fails, an exception is
raised.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(_HERE, "_lib")

T3NS_PREC_FP64 = 0
T3NS_NUM_CONFIGS = 8   # kernel configurations (3, 4: not BF16x3; 5-7: BF16x3 only)
T3NS_PREC_3XTF32 = 1
T3NS_PREC_BF16X3 = 2

_i32p = C.POINTER(C.c_int)
_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


class Ropset(C.Structure):
    _fields_ = [("nrops", C.c_int),
                ("op_nblocks", _i32p),
                ("op_beginblock", C.POINTER(_i32p)),
                ("op_tel", C.POINTER(_f64p))]


class HeffDesc(C.Structure):
    _fields_ = [("isdmrg", C.c_int),
                ("map", C.c_int * 3),
                ("nblocks", C.c_int),
                ("block_off", _i64p),
                ("dims", _i32p),
                ("pair_ptr", _i32p),
                ("pair_old", _i32p),
                ("pair_order", _i32p),
                ("combo_ptr", _i64p),
                ("combo_mpo", _i32p),
                ("combo_sbops", _i32p),
                ("combo_pref", _f64p),
                ("nr_instr", C.c_int),
                ("instr", _i32p),
                ("instr_pref", _f64p),
                ("nrMPOc", C.c_int),
                ("MPOc_beg", _i32p),
                ("ops", Ropset * 3)]


class HeffStats(C.Structure):
    _fields_ = [("size", C.c_int64), ("nblocks", C.c_int64), ("npairs", C.c_int64),
                ("ntasks", C.c_int64), ("flops_ref", C.c_double),
                ("flops_exec", C.c_double), ("bytes_alg", C.c_double),
                ("op_elems", C.c_int64), ("scratch_bytes", C.c_int64)]


class DavidsonInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("max_vecs", C.c_int), ("d_energy", C.c_double),
                ("residual", C.c_double), ("seconds", C.c_double), ("fp64_iterations", C.c_int)]


class RequestResult(C.Structure):
    _fields_ = [("id", C.c_int64), ("status", C.c_int), ("energy", C.c_double),
                ("info", DavidsonInfo), ("bytes", C.c_int64), ("queue_seconds", C.c_double),
                ("run_seconds", C.c_double), ("latency_seconds", C.c_double)]


_lib = None


def load(path: str | None = None):
    """Load ``libt3ns_b200.so`` (raises if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.path.join(LIBDIR, "libt3ns_b200.so")
    if not os.path.exists(p):
        raise RuntimeError(f"engine library not built: {p} (run __graft_entry__.build())")
    lib = C.CDLL(p)
    lib.t3ns_heff_create.argtypes = [C.POINTER(HeffDesc), C.c_int, C.POINTER(C.c_void_p)]
    lib.t3ns_heff_matvec_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.t3ns_heff_matvec_device_per_block.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p,
                                                      C.c_void_p]
    lib.t3ns_heff_matvec_host.argtypes = [C.c_void_p, _f64p, _f64p]
    lib.t3ns_heff_diagonal_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.t3ns_heff_diagonal_host.argtypes = [C.c_void_p, _f64p]
    lib.t3ns_heff_set_precision.argtypes = [C.c_void_p, C.c_int]
    lib.t3ns_heff_set_config.argtypes = [C.c_void_p, C.c_int]
    lib.t3ns_heff_get_config.argtypes = [C.c_void_p]
    lib.t3ns_heff_autotune.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]
    lib.t3ns_heff_get_stats.argtypes = [C.c_void_p, C.POINTER(HeffStats)]
    lib.t3ns_heff_last_launches.argtypes = [C.c_void_p]
    lib.t3ns_heff_check_status.argtypes = [C.c_void_p, C.c_void_p]
    lib.t3ns_heff_destroy.argtypes = [C.c_void_p]
    lib.t3ns_heff_destroy.restype = None
    lib.t3ns_last_error.restype = C.c_char_p
    lib.t3ns_version.restype = C.c_char_p
    if hasattr(lib, "t3ns_davidson_host"):
        lib.t3ns_davidson_host.argtypes = [C.c_void_p, _f64p, _f64p, C.c_int, C.c_int,
                                           C.c_double, C.c_int, _f64p, C.c_void_p]
        lib.t3ns_davidson_device.argtypes = [C.c_void_p, C.c_void_p, _f64p, C.c_int, C.c_int,
                                             C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
    lib.t3ns_precondition_host.argtypes = [C.c_int64, _f64p, C.c_double, _f64p, _f64p]
    lib.t3ns_server_create.argtypes = [C.c_int64, C.c_int, C.POINTER(C.c_void_p)]
    lib.t3ns_server_submit.argtypes = [C.c_void_p, C.POINTER(HeffDesc), C.c_int, _f64p, _f64p,
                                       C.c_double, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_int64)]
    lib.t3ns_server_wait.argtypes = [C.c_void_p, C.c_int64, C.POINTER(RequestResult)]
    lib.t3ns_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                      C.POINTER(C.c_int)]
    lib.t3ns_server_destroy.argtypes = [C.c_void_p]
    lib.t3ns_server_destroy.restype = None
    lib.t3ns_server_estimate_bytes.argtypes = [C.POINTER(HeffDesc), C.c_int, C.c_int]
    lib.t3ns_server_estimate_bytes.restype = C.c_int64
    lib.t3ns_precondition_device_noalloc.argtypes = [C.c_int64, C.c_void_p, C.c_double,
                                                     C.c_void_p, C.c_void_p, C.c_void_p]
    if path is None:
        _lib = lib
    return lib


def check(rc: int, what: str = "call"):
    if rc < 0:
        msg = load().t3ns_last_error().decode(errors="replace")
        raise RuntimeError(f"t3ns {what} failed ({rc}): {msg}")
    return rc


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


class StepDesc:
    """Builds the C descriptor of one step from a step-file record dict and
    keeps every numpy array it points into alive."""

    def __init__(self, s: dict):
        self._keep = []
        keep = self._keep.append
        isd = int(s["isdmrg"][0])
        nb = int(s["nrblocks"][0])
        d = HeffDesc()
        d.isdmrg = isd
        m = self.map_from_step(s)
        for j in range(3):
            d.map[j] = m[j]
        d.nblocks = nb
        bo = np.ascontiguousarray(s["beginblock"].astype(np.int64)); keep(bo)
        d.block_off = _ptr(bo, C.c_int64)
        arrs = {}
        for name, dt in [("sr.dims", np.int32), ("sr.pair_ptr", np.int32),
                         ("sr.pair_old", np.int32), ("sr.pair_order", np.int32),
                         ("sr.combo_ptr", np.int64), ("sr.combo_mpo", np.int32),
                         ("sr.combo_sbops", np.int32), ("sr.combo_pref", np.float64),
                         ("iset.instr", np.int32), ("iset.pref", np.float64),
                         ("iset.MPOc_beg", np.int32)]:
            a = np.ascontiguousarray(s[name].astype(dt))
            if a.size == 0:
                a = np.zeros(1, dt)
            keep(a)
            arrs[name] = a
        d.dims = _ptr(arrs["sr.dims"], C.c_int)
        d.pair_ptr = _ptr(arrs["sr.pair_ptr"], C.c_int)
        d.pair_old = _ptr(arrs["sr.pair_old"], C.c_int)
        d.pair_order = _ptr(arrs["sr.pair_order"], C.c_int)
        d.combo_ptr = _ptr(arrs["sr.combo_ptr"], C.c_int64)
        d.combo_mpo = _ptr(arrs["sr.combo_mpo"], C.c_int)
        d.combo_sbops = _ptr(arrs["sr.combo_sbops"], C.c_int)
        d.combo_pref = _ptr(arrs["sr.combo_pref"], C.c_double)
        d.nr_instr = int(s["iset.nr_instr"][0])
        d.instr = _ptr(arrs["iset.instr"], C.c_int)
        d.instr_pref = _ptr(arrs["iset.pref"], C.c_double)
        d.nrMPOc = int(s["iset.nrMPOc"][0])
        d.MPOc_beg = _ptr(arrs["iset.MPOc_beg"], C.c_int)
        for i in range(2 if isd else 3):
            self._fill_ropset(d.ops[i], s, i)
        self.desc = d
        self.size = int(bo[-1])

    @staticmethod
    def map_from_step(s: dict):
        """Memory-axis -> operator map (reference make_map, src/Heff.c:668-682)."""
        if int(s["isdmrg"][0]):
            return [0, 1, 2]
        ros = s["rOperators_on_site"]
        posB = int(s["posB"][0])
        swap = ros[1] != posB and ros[0] == posB
        return [1, 0, 2] if swap else [0, 1, 2]

    def _fill_ropset(self, rs: Ropset, s: dict, i: int):
        keep = self._keep.append
        nrops = int(s[f"ops{i}.nrops"][0])
        rs.nrops = nrops
        if nrops == 0:
            return
        hss = s[f"ops{i}.hss_of_ops"]
        bbh = s[f"ops{i}.begin_blocks_of_hss"]
        bb = np.ascontiguousarray(s[f"ops{i}.beginblock"].astype(np.int32)); keep(bb)
        tel = np.ascontiguousarray(s[f"ops{i}.tel"]); keep(tel)
        nbl = (bbh[hss + 1] - bbh[hss]).astype(np.int32); keep(nbl)
        bb_ptrs = (_i32p * nrops)()
        tel_ptrs = (_f64p * nrops)()
        boff = 0
        toff = 0
        for k in range(nrops):
            n = int(nbl[k])
            bb_ptrs[k] = C.cast(bb.ctypes.data + 4 * boff, _i32p)
            tel_ptrs[k] = C.cast(tel.ctypes.data + 8 * toff, _f64p)
            toff += int(bb[boff + n])
            boff += n + 1
        keep(bb_ptrs)
        keep(tel_ptrs)
        rs.op_nblocks = _ptr(nbl, C.c_int)
        rs.op_beginblock = bb_ptrs
        rs.op_tel = tel_ptrs


class HeffPlan:
    """Owner of one engine plan (t3ns_heff)."""

    def __init__(self, desc: StepDesc, precision: int = T3NS_PREC_FP64):
        self.lib = load()
        self._desc = desc
        h = C.c_void_p()
        check(self.lib.t3ns_heff_create(C.byref(desc.desc), precision, C.byref(h)), "heff_create")
        self.h = h
        st = HeffStats()
        check(self.lib.t3ns_heff_get_stats(self.h, C.byref(st)), "get_stats")
        self.stats = {f: getattr(st, f) for f, _ in HeffStats._fields_}
        self.size = int(st.size)

    def matvec_host(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        check(self.lib.t3ns_heff_matvec_host(self.h, _ptr(x, C.c_double), _ptr(y, C.c_double)),
              "matvec_host")
        return y

    def set_precision(self, precision: int):
        check(self.lib.t3ns_heff_set_precision(self.h, precision), "set_precision")

    def set_config(self, config: int):
        check(self.lib.t3ns_heff_set_config(self.h, config), "set_config")

    def config(self) -> int:
        return int(self.lib.t3ns_heff_get_config(self.h))

    def autotune(self, reps: int = 2, force: bool = True):
        """Time every kernel configuration and keep the fastest; returns the
        median milliseconds per configuration (0 where not timed)."""
        ms = (C.c_double * 16)()
        check(self.lib.t3ns_heff_autotune(self.h, reps, int(force), ms), "autotune")
        return [ms[i] for i in range(T3NS_NUM_CONFIGS)]

    def matvec_device(self, x_ptr: int, y_ptr: int, stream: int = 0):
        check(self.lib.t3ns_heff_matvec_device(self.h, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                               C.c_void_p(stream)), "matvec_device")

    def matvec_device_per_block(self, x_ptr: int, y_ptr: int, stream: int = 0):
        """The same product with one kernel launch per output block."""
        check(self.lib.t3ns_heff_matvec_device_per_block(self.h, C.c_void_p(x_ptr),
                                                         C.c_void_p(y_ptr), C.c_void_p(stream)),
              "matvec_device_per_block")

    def diagonal_host(self) -> np.ndarray:
        d = np.empty(self.size)
        check(self.lib.t3ns_heff_diagonal_host(self.h, _ptr(d, C.c_double)), "diagonal_host")
        return d

    def davidson_host(self, result: np.ndarray, diagonal: np.ndarray, tol: float = 1e-5,
                      max_its: int = 100, max_vecs: int = 30, keep: int = 2):
        """Lowest eigenpair; ``result`` (guess) is overwritten with the vector.
        Returns ``(energy, return_code, info)``."""
        assert result.dtype == np.float64 and result.flags.c_contiguous
        diagonal = np.ascontiguousarray(diagonal, dtype=np.float64)
        e = C.c_double()
        info = DavidsonInfo()
        rc = check(self.lib.t3ns_davidson_host(self.h, _ptr(result, C.c_double), C.byref(e),
                                                max_vecs, keep, tol, max_its,
                                                _ptr(diagonal, C.c_double), C.byref(info)),
                   "davidson_host")
        return e.value, rc, {f: getattr(info, f) for f, _ in DavidsonInfo._fields_}

    def last_launches(self) -> int:
        return int(self.lib.t3ns_heff_last_launches(self.h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.t3ns_heff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
