"""include/fourphonon_b200.f90, the Fortran host's ISO_C_BINDING module (CPU).

No Fortran compiler is installed here, so this checks the module's structure:
it is the generator's current output for the header, every C entry point has
one bind(c) interface with the same name and argument count, the kinds follow
the C types, and every line fits free-form Fortran's 132 columns.
"""
import os
import re
import subprocess
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "include"))
import make_fortran_module as M  # noqa: E402


def _module():
    return open(os.path.join(ROOT, "include", "fourphonon_b200.f90")).read()


def test_module_is_current():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "include", "make_fortran_module.py"), "--check"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_every_entry_point_has_an_interface():
    header = open(M.HEADER).read()
    mod = _module()
    joined = re.sub(r"&\n\s*", "", mod)  # undo the continuation lines
    protos = M.prototypes(header)
    assert len(protos) >= 40
    for ret, name, params in protos:
        m = re.search(rf"function {name}\(([^)]*)\) bind\(c, name=\"{name}\"\)", joined)
        assert m, name
        args = [a.strip() for a in m.group(1).split(",")]
        assert args == [p[1] for p in params], name
        body = joined[m.end():joined.index(f"end function {name}", m.end())]
        for ctype, pname, extent in params:
            decl = re.search(rf"\n\s*(.*) :: {pname}\b", body)
            assert decl, (name, pname)
            d = decl.group(1)
            base = ctype.replace("const ", "").replace("*", "").strip()
            device = name in M.DEVICE_POINTERS and "*" in ctype and base != "fp4_globals"
            if base == "fp4_globals":  # a host record in every entry point
                assert d.startswith("type(fp4_globals)"), (name, pname, d)
            elif base in ("fp4_ctx", "fp4_server", "void") or device:
                assert d.startswith("type(c_ptr)"), (name, pname, d)
            elif pname == "eigenvect":
                assert d.startswith("complex(c_double_complex)"), (name, pname, d)
            else:
                assert d.startswith(M.KIND[base]), (name, pname, d)
            by_value = ("*" not in ctype and extent is None) \
                or (base in ("fp4_ctx", "fp4_server", "void") and ctype.count("*") == 1) \
                or device
            assert ("value" in d) == by_value, (name, pname, d)


def test_line_lengths_and_blocks():
    mod = _module()
    assert all(len(x) <= 132 for x in mod.splitlines())
    assert mod.count("\n     end function ") == len(M.prototypes(open(M.HEADER).read()))
    assert "module fp4_b200" in mod and mod.rstrip().endswith("end module fp4_b200")
    for name, value in M.constants(open(M.HEADER).read()):
        assert f"integer(c_int), parameter :: {name} = {value}" in mod
