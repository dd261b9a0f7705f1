"""The C-ABI library loads and exports every entry point the public header
declares; without a GPU the device entry points fail with a status code
instead of crashing or blocking."""
import ctypes as C

import pytest


def test_exports_match_header():
    import cfdfs
    L = cfdfs.lib()
    names = cfdfs.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.cfd_abi_version() == 1


def test_default_options():
    import cfdfs
    o = cfdfs.default_options()
    assert o.precision == cfdfs.FP64 and o.cg_rtol == 1e-8 and o.cg_maxit == 1000 and o.cg_warm == 0


def test_null_arguments_are_rejected():
    import cfdfs
    L = cfdfs.lib()
    assert L.cfd_step0(None) == cfdfs.CFD_E_BADARG
    assert L.cfd_run(None, 1, None) == cfdfs.CFD_E_BADARG
    assert L.cfd_load_inp(None, b"x") == cfdfs.CFD_E_BADARG
    assert L.cfdh_load(None, b"x", None, 0) == cfdfs.CFD_E_BADARG


def test_create_without_gpu_returns_status():
    import torch
    import cfdfs
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = cfdfs.lib().cfd_create(C.byref(h), 0)
    assert rc == cfdfs.CFD_E_CUDA and not h.value


def test_integration_example_compiles(tmp_path):
    """The C++ integration example of INTEGRATION.md (the branch a maintainer
    adds beside USECUDA in the reference's time loop) compiles against
    include/cfdfs.h: every call and argument it shows exists in the header."""
    import os
    import re
    import shutil
    import subprocess
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    text = open(os.path.join(root, "INTEGRATION.md")).read()
    snip = re.search(r"```cpp\n(.*?)```", text, re.S).group(1)
    body = snip.replace("#ifdef USE_CFDFS\n", "").replace("#endif\n", "")
    head, rest = body.split("// in main(), replacing selectCUDAdevice():", 1)
    head = head.replace('#include "cfdfs.h"', "#include <cstdio>\n#include <cstdlib>\n#include <string>\n"
                                              '#include "cfdfs.h"')
    # the reference's own variables the example uses
    globs = ("static std::string whichProblem;\n"
             "static int maxIter = 4, monPoint = 0, iter = 0, checkAccConvergence = 0;\n"
             "static double tolerance = 1e-3, convergenceCriteria = 1e-6, maxAcc = 0;\n")
    src = tmp_path / "example.cpp"
    src.write_text(head + globs + "void timeLoopBody() {\n" + rest + "}\n")
    r = subprocess.run([gxx, "-std=c++17", "-Wall", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(root, "include"), str(src)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
