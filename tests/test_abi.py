"""CPU checks of the C ABI: both libraries load, every function declared in
include/*.h is exported, and the ctypes mirror has the C layouts."""
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADERS = {"hacapk_b200.h": "ENGINE_LIB", "hacapk_b200_build.h": "BUILD_LIB"}


def declared_functions(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = re.sub(r"//[^\n]*", "", src)
    src = re.sub(r"typedef\s+struct\s+\w*\s*\{.*?\}\s*\w+\s*;", "", src, flags=re.S)
    src = re.sub(r"typedef[^;]*;", "", src)
    src = re.sub(r"enum\s*\w*\s*\{.*?\}\s*;", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_]\w*)\s*\([^;{)]*\)\s*;", src)))


@pytest.mark.parametrize("header", sorted(HEADERS))
def test_every_declared_symbol_is_exported(build_libs, header):
    from hacapk_b200 import abi
    lib = getattr(abi, HEADERS[header])
    names = declared_functions(header)
    assert len(names) >= 8
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    missing = [n for n in names if n not in exported]
    assert not missing, f"{header}: not exported by {os.path.basename(lib)}: {missing}"


def test_engine_library_exports_only_its_c_abi(build_libs):
    """The engine library's dynamic symbol table is exactly the functions of
    include/hacapk_b200.h (the export map keeps the C++ internals local), so
    a Fortran application linking it sees no other names."""
    from hacapk_b200 import abi
    out = subprocess.run(["nm", "-D", "--defined-only", abi.ENGINE_LIB], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if line.strip()}
    assert exported == set(declared_functions("hacapk_b200.h"))


def test_libraries_load_without_a_gpu(build_libs):
    from hacapk_b200 import abi
    abi.engine_lib()
    abi.build_lib()


def test_ctypes_layouts_match_c(build_libs, tmp_path):
    import ctypes as C
    from hacapk_b200 import abi
    prog = tmp_path / "layout.c"
    prog.write_text('''#include <stdio.h>
#include <stddef.h>
#include "hacapk_b200_build.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(stc_HACApK_leafmtx), sizeof(stc_HACApK_leafmtxp),
         offsetof(stc_HACApK_leafmtxp, st_lf), sizeof(stc_HACApK_lcontrol), sizeof(hbx_options), sizeof(hbx_info),
         sizeof(hbx_solve_opts), sizeof(hbx_solve_info), sizeof(hbx_build_params), sizeof(hbx_build_stats),
         offsetof(hbx_solve_info, launches));
  return 0; }''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(prog)], check=True)
    got = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()))
    want = [C.sizeof(abi.LeafMtx), C.sizeof(abi.LeafMtxP), abi.LeafMtxP.st_lf.offset, C.sizeof(abi.LControl),
            C.sizeof(abi.Options), C.sizeof(abi.Info), C.sizeof(abi.SolveOpts), C.sizeof(abi.SolveInfo),
            C.sizeof(abi.BuildParams), C.sizeof(abi.BuildStats), abi.SolveInfo.launches.offset]
    assert got == want


def test_engine_library_has_no_cpu_compute_fallback(build_libs):
    """The engine library links only the CUDA runtime and the host planner;
    the CPU matvec of the oracle is not part of it."""
    from hacapk_b200 import abi
    out = subprocess.run(["nm", "-D", abi.ENGINE_LIB], capture_output=True, text=True, check=True).stdout
    assert "orc_" not in out and "c_hacapk_adot_body_lfmtx_" not in [l.split()[-1] for l in out.splitlines()]


def test_unknown_precision_is_refused(build_libs):
    """An unknown storage precision is refused before any CUDA call."""
    from conftest import sphere
    from hacapk_b200.engine import Engine, HbxError
    from hacapk_b200 import abi
    H = sphere(2)
    with pytest.raises(HbxError) as e:
        Engine(H.st, H.nd, precision=7)
    assert abi.STATUS[e.value.status] == "HBX_ERR_UNSUPPORTED"
