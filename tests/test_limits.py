"""Host-side limits of the matvec plan (no GPU): the kernels address
elements inside one block with 32-bit offsets, so a block of 2^31 or more
elements is rejected at plan build with T3NS_E_LIMIT instead of being read
out of bounds later."""
import ctypes as C

import numpy as np

from t3ns_b200 import native

T3NS_E_LIMIT = -4


def _desc(dims):
    """A descriptor of one block of the given dims and no pairs (nothing to
    contract); the arrays are kept on the returned object."""
    d = native.HeffDesc()
    d.isdmrg = 0
    for j in range(3):
        d.map[j] = j
    d.nblocks = 1
    keep = {
        "off": np.array([0, int(np.prod(np.array(dims, dtype=np.int64)))], np.int64),
        "dims": np.array(dims, np.int32),
        "pair_ptr": np.zeros(2, np.int32),
        "i32": np.zeros(4, np.int32),
        "i64": np.zeros(2, np.int64),
        "f64": np.zeros(2),
        "beg": np.zeros(2, np.int32),
    }
    i32p, i64p, f64p = C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_double)
    d.block_off = keep["off"].ctypes.data_as(i64p)
    d.dims = keep["dims"].ctypes.data_as(i32p)
    d.pair_ptr = keep["pair_ptr"].ctypes.data_as(i32p)
    d.pair_old = d.pair_order = d.combo_mpo = d.combo_sbops = d.instr = keep["i32"].ctypes.data_as(i32p)
    d.combo_ptr = keep["i64"].ctypes.data_as(i64p)
    d.combo_pref = d.instr_pref = keep["f64"].ctypes.data_as(f64p)
    d.nr_instr = 0
    d.nrMPOc = 0
    d.MPOc_beg = keep["beg"].ctypes.data_as(i32p)
    for i in range(3):
        d.ops[i].nrops = 0
    return d, keep


def _plan_dump(d, tmp_path):
    lib = native.load()
    lib.t3ns_heff_plan_dump_config.argtypes = [C.POINTER(native.HeffDesc), C.c_int, C.c_char_p]
    return lib.t3ns_heff_plan_dump_config(C.byref(d), 0, str(tmp_path / "p.t3c").encode())


def test_block_of_2_to_the_31_elements_is_rejected(tmp_path):
    d, keep = _desc([2048, 1024, 1024])
    assert _plan_dump(d, tmp_path) == T3NS_E_LIMIT
    assert b"2^31" in native.load().t3ns_last_error()


def test_block_just_below_the_limit_is_accepted(tmp_path):
    d, keep = _desc([2047, 1024, 1024])
    assert _plan_dump(d, tmp_path) == 0
