"""The diagnostic channel (no GPU): with a prefix set by trl_set_debug,
trl_print_info and trl_terse_info append to the per-process file
prefix + rank (the reference's trl_reopen_logfile, SRC/trlaux.c:86-118)
instead of stdout; without one they write to stdout."""
import ctypes as C

from nutrlan_b200 import TrlInfo


def test_print_info_goes_to_the_log_file(lib, tmp_path, capfd):
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), 1000, 40, -1, 8, 1e-8, 1, 1000, None)
    prefix = str(tmp_path / "LOG_run")
    lib.trl_set_debug(C.byref(info), 0, prefix.encode())
    capfd.readouterr()
    lib.trl_print_info(C.byref(info), 3000)
    lib.trl_terse_info(C.byref(info), None)
    C.CDLL(None).fflush(None)
    out = capfd.readouterr().out
    text = (tmp_path / "LOG_run0").read_text()
    assert "TRLAN execution summary" in text and "MAXLAN:" in text
    assert "TRLAN execution summary" not in out
    info2 = TrlInfo()
    lib.trl_init_info(C.byref(info2), 1000, 40, -1, 8, 1e-8, 1, 1000, None)
    lib.trl_print_info(C.byref(info2), 3000)
    C.CDLL(None).fflush(None)
    assert "TRLAN execution summary" in capfd.readouterr().out
