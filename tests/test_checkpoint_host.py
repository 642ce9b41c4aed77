"""Host side of the checkpoint channel (no GPU): trl_set_iguess with
guess > 1 checks that the per-process file of the reference's naming
(prefix up to the first blank + rank, zero-padded to the digits of npes)
exists, and trl_set_checkpoint stores the prefix."""
import ctypes as C

from nutrlan_b200 import TrlInfo


def test_iguess_checks_reference_file_name(lib, tmp_path):
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), 1000, 40, -1, 8, 1e-8, 1, 1000, None)
    prefix = str(tmp_path / "cpt")
    lib.trl_set_iguess(C.byref(info), 0, 2, 0, prefix.encode())
    assert info.stat == -8 and info.guess == 2
    (tmp_path / "cpt0").write_bytes(b"\0" * 8)
    lib.trl_set_iguess(C.byref(info), 0, 2, 0, prefix.encode())
    assert info.stat == 0
    # With 12 processes the rank is written with two digits.
    info.npes, info.my_pe = 12, 3
    lib.trl_set_iguess(C.byref(info), 0, 2, 0, prefix.encode())
    assert info.stat == -8
    (tmp_path / "cpt03").write_bytes(b"\0" * 8)
    lib.trl_set_iguess(C.byref(info), 0, 2, 0, prefix.encode())
    assert info.stat == 0
    # Only the part before the first blank names the file.
    lib.trl_set_iguess(C.byref(info), 0, 2, 0, (prefix + " ignored").encode())
    assert info.stat == 0


def test_set_checkpoint_stores_prefix(lib):
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), 1000, 40, -1, 8, 1e-8, 1, 1000, None)
    lib.trl_set_checkpoint(C.byref(info), 4, b"/tmp/cp_prefix")
    assert info.cpflag == 4 and bytes(info.cpfile).split(b"\0")[0] == b"/tmp/cp_prefix"
