"""ctypes description of the C ABI shared by libtrlan_b200.so and nuTRLan.

``TrlInfo`` mirrors ``trl_info`` field for field (reference INC/trlan.h:77-245,
800 bytes on LP64), so the same Python object can be handed to the B200
library and to the reference library built under ``oracle/_ref``.
"""
import ctypes as C

c_int, c_double, c_void_p, c_long = C.c_int, C.c_double, C.c_void_p, C.c_long

_FIELDS = [
    ("stat", c_int), ("lohi", c_int), ("ned", c_int), ("nec", c_int),
    ("tol", c_double), ("mpicomp", c_void_p),
    ("maxlan", c_int), ("klan", c_int), ("maxmv", c_int), ("restart", c_int),
    ("locked", c_int), ("guess", c_int), ("matvec", c_int), ("nloop", c_int),
    ("north", c_int), ("nrand", c_int), ("flop", c_int), ("flop_h", c_int),
    ("flop_r", c_int),
    ("rflp", c_double), ("rflp_h", c_double), ("rflp_r", c_double),
    ("clk_rate", c_long), ("clk_max", c_long), ("clk_tot", c_long),
    ("clk_op", c_long), ("clk_orth", c_long), ("clk_res", c_long),
    ("tick_t", c_double), ("tick_o", c_double), ("tick_h", c_double),
    ("tick_r", c_double),
    ("clk_in", c_int), ("wrds_in", c_int), ("clk_out", c_int),
    ("wrds_out", c_int),
    ("anrm", c_double),
    ("my_pe", c_int), ("npes", c_int), ("nloc", c_int), ("ntot", c_int),
    ("verbose", c_int),
    ("crat", c_double), ("trgt", c_double), ("tres", c_double),
    ("tmv", c_int), ("avgm", c_double),
    ("cfac", c_double), ("ptres", c_double), ("predicted_crate", c_double),
    ("mgap", c_double), ("mgamma", c_double), ("gamma0", c_double),
    ("old_target", c_double),
    ("target_id", c_int), ("old_locked", c_int), ("k1", c_int), ("k2", c_int),
    ("k", c_int), ("rfact", c_double), ("ref", c_double),
    ("log_io", c_int), ("log_fp", c_void_p), ("log_file", C.c_char * 128),
    ("cpflag", c_int), ("cpio", c_int), ("cpt_fp", c_void_p),
    ("cpfile", C.c_char * 128), ("oldcpf", C.c_char * 128),
    ("mvparam", c_void_p),
]


class TrlInfo(C.Structure):
    _fields_ = _FIELDS


class TrlDComplex(C.Structure):
    _fields_ = [("r", c_double), ("i", c_double)]


assert C.sizeof(TrlInfo) == 800, C.sizeof(TrlInfo)
assert TrlInfo.mvparam.offset == 792

DP = C.POINTER(c_double)
ZP = C.POINTER(TrlDComplex)

# void op(int nrow, int ncol, const double *x, int ldx, double *y, int ldy, void *mvparam)
MATVEC = C.CFUNCTYPE(None, c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p)
# void user_ortho(int nrow, double *v, double *normDiff)
USER_ORTHO = C.CFUNCTYPE(None, c_int, c_void_p, c_void_p)


def declare_common(lib):
    """Prototypes of the entry points both libraries export."""
    lib.trl_init_info.argtypes = [C.POINTER(TrlInfo), c_int, c_int, c_int, c_int,
                                  c_double, c_int, c_int, c_void_p]
    lib.trl_init_info.restype = None
    lib.trl_set_iguess.argtypes = [C.POINTER(TrlInfo), c_int, c_int, c_int, C.c_char_p]
    lib.trl_set_iguess.restype = None
    lib.trl_set_restart.argtypes = [C.POINTER(TrlInfo), c_double]
    lib.trl_set_restart.restype = None
    lib.trl_set_debug.argtypes = [C.POINTER(TrlInfo), c_int, C.c_char_p]
    lib.trl_set_debug.restype = None
    lib.trl_set_checkpoint.argtypes = [C.POINTER(TrlInfo), c_int, C.c_char_p]
    lib.trl_set_checkpoint.restype = None
    lib.trlan.argtypes = [MATVEC, C.c_void_p, C.POINTER(TrlInfo), c_int, c_int,
                          c_void_p, c_void_p, c_int, c_int, c_void_p]
    lib.trlan.restype = None
    lib.ztrlan.argtypes = [MATVEC, C.POINTER(TrlInfo), c_int, c_int, c_void_p,
                           c_void_p, c_int, c_void_p, c_int, c_void_p, c_int]
    lib.ztrlan.restype = None
    lib.trl_print_info.argtypes = [C.POINTER(TrlInfo), c_int]
    lib.trl_print_info.restype = None
    lib.trl_terse_info.argtypes = [C.POINTER(TrlInfo), c_void_p]
    lib.trl_terse_info.restype = None
    lib.trl_check_ritz.argtypes = [MATVEC, C.POINTER(TrlInfo), c_int, c_int, c_void_p,
                                   c_int, c_void_p, C.POINTER(c_int), c_void_p,
                                   c_void_p, c_void_p, c_int]
    lib.trl_check_ritz.restype = None
    lib.ztrl_check_ritz.argtypes = [MATVEC, C.POINTER(TrlInfo), c_int, c_int, c_void_p,
                                    c_int, c_void_p, C.POINTER(c_int), c_void_p,
                                    c_void_p, c_void_p, c_int]
    lib.ztrl_check_ritz.restype = None
    lib.trl_rayleigh_quotients.argtypes = [MATVEC, C.POINTER(TrlInfo), c_int, c_void_p,
                                           c_int, c_void_p, c_void_p]
    lib.trl_rayleigh_quotients.restype = None
    lib.trl_ritz_projection.argtypes = [MATVEC, C.POINTER(TrlInfo), c_int, c_void_p,
                                        c_int, c_void_p, c_void_p, c_int, c_void_p]
    lib.trl_ritz_projection.restype = None
