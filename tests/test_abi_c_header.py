"""The C-ABI as a C caller (or a Fortran bind(C) interface) sees it (CPU).

* include/fourphonon_b200.h compiles as strict C99 with every warning an
  error, so a C or Fortran host can include it without a C++ compiler;
* a C program links against libfp4b200.so and resolves every declared entry
  point;
* the fp4_globals record has the same field offsets and size in C as in the
  ctypes binding (a Fortran `type, bind(c)` with the fields in header order
  gets the C layout);
* fp4_create without a CUDA device returns an error code instead of crashing.
"""
import ctypes as ct
import os
import re
import shutil
import subprocess

import pytest

from fourphonon_b200 import abi

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
FIELDS = ("ngrid", "nbands", "rlattvec", "T", "scalebroad", "omega_max", "onlyharmonic", "nelements", "natoms",
          "masses", "types")


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "fourphonon_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fp4_[a-z0-9_]+)\s*\(", src)))


def _program(symbols):
    refs = "\n".join(f"    (entry_point)&{s}," for s in symbols)
    offs = "\n".join(f'    printf("{f} %zu\\n", offsetof(fp4_globals, {f}));' for f in FIELDS)
    return f"""#include <stddef.h>
#include <stdio.h>
#include "fourphonon_b200.h"

typedef void (*entry_point)(void);
static const entry_point entry_points[] = {{
{refs}
}};

int main(void) {{
    fp4_ctx *ctx = NULL;
    int rc;
    printf("size %zu\\n", sizeof(fp4_globals));
{offs}
    printf("entry_points %zu\\n", sizeof entry_points / sizeof entry_points[0]);
    rc = fp4_create(&ctx, 0);
    if (rc == FP4_OK) {{
        fp4_destroy(ctx);
        printf("create device\\n");
    }} else {{
        printf("create %d\\n", rc);
    }}
    return 0;
}}
"""


@pytest.fixture(scope="module")
def c_run(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    lib = abi.load(build_if_missing=True)  # builds the library when it is absent
    assert lib is not None
    libdir = os.path.dirname(abi.library_path())
    d = tmp_path_factory.mktemp("cabi")
    src = d / "caller.c"
    exe = d / "caller"
    src.write_text(_program(declared_symbols()))
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
           str(src), "-o", str(exe), "-L", libdir, "-lfp4b200", f"-Wl,-rpath,{libdir}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    vals = {}
    for line in out.stdout.splitlines():
        k, v = line.split()
        vals[k] = v
    return vals


def test_header_is_strict_c99_and_links(c_run):
    assert int(c_run["entry_points"]) == len(declared_symbols())


def test_globals_layout_matches_the_binding(c_run):
    assert int(c_run["size"]) == ct.sizeof(abi.Globals)
    for f in FIELDS:
        assert int(c_run[f]) == getattr(abi.Globals, f).offset, f


def test_create_from_c_without_device(c_run):
    if "device" in c_run:
        pytest.skip("a CUDA device is present")
    assert int(c_run["create"]) in (-1, -2)  # FP4_E_ARG or FP4_E_CUDA
