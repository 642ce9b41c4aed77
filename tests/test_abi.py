"""The C-ABI library loads without a GPU and exports every declared symbol;
trl_info keeps the reference's layout."""
import ctypes as C
import os
import re
import subprocess

import pytest

from nutrlan_b200 import TrlInfo, LIB_PATH

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("trlan.h", "ztrlan.h", "trlx.h", "ftrlan.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b([a-z_][a-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("trl", "ztrl")) and name not in ("trl_matvec", "trl_uo", "ztrl_matvec", "trl_fmatvec",
                                                                 "ztrl_fmatvec"):
                names.add(name)
    return names


def test_library_loads_and_exports_all_declared_symbols(lib):
    names = declared_functions()
    assert "trlan" in names and "ztrlan" in names and "trlx_trlan" in names
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = sorted(n for n in names if n not in exported)
    assert not missing, missing
    for n in names:
        getattr(lib, n)


def test_trl_info_layout_matches_reference_header():
    assert C.sizeof(TrlInfo) == 800
    assert TrlInfo.mvparam.offset == 792
    assert TrlInfo.clk_rate.offset == 112
    assert TrlInfo.anrm.offset == 208
    assert TrlInfo.log_file.offset == 392


def test_header_compiles_and_layout_in_c(tmp_path):
    src = tmp_path / "abi.c"
    src.write_text(
        "#include <stddef.h>\n#include <stdio.h>\n#include \"trlx.h\"\n"
        "int main(){printf(\"%zu %zu\\n\", sizeof(trl_info), offsetof(trl_info, mvparam));"
        "return 0;}\n")
    exe = tmp_path / "abi"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert out == ["800", "792"]


def test_init_info_defaults(lib):
    info = TrlInfo()
    lib.trl_init_info(C.byref(info), 1000, 50, -1, 5, 0.0, 0, 0, None)
    assert info.tol == pytest.approx(1.4901161193847656e-08)
    assert info.restart == 0 and info.maxlan == 50 and info.ned == 5
    assert info.maxmv == 1000 and info.ntot == 1000 and info.nloc == 1000
    assert info.trgt < -1e300 and info.tres == -1.0 and info.crat == 1.0 and info.tmv == -1
    # tol > 1 is read as a reciprocal, tol tiny becomes eps
    lib.trl_init_info(C.byref(info), 1000, 3, 1, 5, 50.0, 7, 100, None)
    assert info.tol == pytest.approx(0.02) and info.maxlan == 11 and info.restart == 7


def test_version_string(lib):
    assert b"sm_100a" in lib.trlx_version()


REF_ROOT = os.environ.get("TRLAN_REFERENCE", "/root/reference")


@pytest.mark.skipif(not os.path.isfile(os.path.join(REF_ROOT, "INC", "trlan.h")),
                    reason="reference headers not present (set TRLAN_REFERENCE)")
def test_every_trl_info_offset_matches_the_reference_header(tmp_path):
    """sizeof(trl_info) and offsetof of every field, compiled with gcc
    against include/trlan.h and against the reference's INC/trlan.h
    (:77-245), are identical."""
    fields = [f[0] for f in TrlInfo._fields_]
    body = "".join(f'printf("{f} %zu\\n", offsetof(trl_info, {f}));' for f in fields)
    src = tmp_path / "offsets.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"trlan.h\"\n"
                   "int main(){printf(\"sizeof %zu\\n\", sizeof(trl_info));" + body + "return 0;}\n")
    outs = []
    for inc in (os.path.join(ROOT, "include"), os.path.join(REF_ROOT, "INC")):
        exe = tmp_path / ("off_" + str(len(outs)))
        subprocess.run(["gcc", "-I", inc, str(src), "-o", str(exe)], check=True)
        outs.append(subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout)
    assert outs[0] == outs[1]
    got = dict(line.split() for line in outs[0].splitlines())
    assert got["sizeof"] == "800" and len(got) == len(fields) + 1
    for f in fields:                      # and the Python mirror agrees with both
        assert int(got[f]) == getattr(TrlInfo, f).offset, f


def _mirrors():
    from nutrlan_b200._lib import TrlxStats, TrlxOptions, TrlxTuneResult
    from nutrlan_b200.batched import BatchOptions, BatchConfig
    return {"trlx_stats": TrlxStats, "trlx_options": TrlxOptions, "trlx_tune_result": TrlxTuneResult,
            "trlx_batch_options": BatchOptions, "trlx_batch_config": BatchConfig}


def test_trlx_struct_mirrors_match_the_header(tmp_path):
    """Every ctypes mirror of a trlx.h struct has the C compiler's size and
    field offsets (fields appended to a struct keep the earlier offsets)."""
    mirrors = _mirrors()
    lines = []
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, *_ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    src = tmp_path / "mirrors.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"trlx.h\"\nint main(){\n"
                   + "\n".join(lines) + "\nreturn 0;}\n")
    exe = tmp_path / "mirrors"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        cname, key, val = ln.split()
        got[(cname, key)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for fname, *_ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)
