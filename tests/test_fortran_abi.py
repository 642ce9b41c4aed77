"""Fortran-callable entry points (include/ftrlan.h) on the host: every
argument is passed by reference, CHARACTER arguments arrive blank-padded
with their lengths after the other arguments, as a Fortran compiler passes
them.  The solver entry points are exercised in tests/test_gpu_fortran.py."""
import ctypes as C

from nutrlan_b200 import TrlInfo

P = C.POINTER


def _declare(lib):
    lib.trl_init_info_.argtypes = [P(TrlInfo), P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_int), P(C.c_double),
                                   P(C.c_int), P(C.c_int)]
    lib.trl_set_checkpoint_.argtypes = [P(TrlInfo), P(C.c_int), C.c_char_p, C.c_size_t]
    lib.trl_set_iguess_.argtypes = [P(TrlInfo), P(C.c_int), P(C.c_int), P(C.c_int), C.c_char_p, C.c_size_t]
    lib.trl_set_restart_.argtypes = [P(TrlInfo), P(C.c_double)]
    for f in (lib.trl_init_info_, lib.trl_set_checkpoint_, lib.trl_set_iguess_, lib.trl_set_restart_):
        f.restype = None
    return lib


def _i(v):
    return C.byref(C.c_int(v))


def test_init_info_by_reference_matches_c_entry(lib):
    _declare(lib)
    a, b = TrlInfo(), TrlInfo()
    lib.trl_init_info_(C.byref(a), _i(5000), _i(60), _i(-1), _i(12), C.byref(C.c_double(1e-9)), _i(3), _i(4000))
    lib.trl_init_info(C.byref(b), 5000, 60, -1, 12, 1e-9, 3, 4000, None)
    assert bytes(a) == bytes(b)
    lib.trl_set_restart_(C.byref(a), C.byref(C.c_double(1.7)))
    assert a.rfact == 1.7


def test_blank_padded_character_arguments(lib, tmp_path):
    _declare(lib)
    info = TrlInfo()
    lib.trl_init_info_(C.byref(info), _i(1000), _i(40), _i(-1), _i(8), C.byref(C.c_double(1e-8)), _i(1),
                       _i(1000))
    prefix = str(tmp_path / "fcp")
    padded = (prefix + " " * 20).encode()
    lib.trl_set_checkpoint_(C.byref(info), _i(2), padded, len(padded))
    assert info.cpflag == 2 and bytes(info.cpfile).split(b"\0")[0] == prefix.encode()
    # iguess > 1 checks that <prefix><rank> exists; the padding is not part of it.
    lib.trl_set_iguess_(C.byref(info), _i(0), _i(2), _i(1), padded, len(padded))
    assert info.stat == -8 and info.guess == 2
    (tmp_path / "fcp0").write_bytes(b"\0" * 8)
    lib.trl_set_iguess_(C.byref(info), _i(0), _i(2), _i(1), padded, len(padded))
    assert info.stat == 0
