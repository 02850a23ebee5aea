#!/usr/bin/env python
"""Writes include/fourphonon_b200.f90, the ISO_C_BINDING interface module of
every entry point declared in include/fourphonon_b200.h, for the Fortran host
(ShengBTE.f90) to `use`.

Each C prototype becomes one `bind(c)` interface with the same name and
arguments.  Host arrays become assumed-size dummies of the matching kind
(eigenvect as complex(c_double_complex)); scalars passed by value get the
`value` attribute; opaque handles, streams and the device pointers of the
allocation-free entry point are type(c_ptr); the scalar results that a few
calls return through pointers are scalar dummies.  fp4_globals is declared
as a bind(c) derived type with the header's fields in order.

    python include/make_fortran_module.py          # (re)write the module
    python include/make_fortran_module.py --check  # exit 1 if it is stale
"""
from __future__ import annotations

import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "fourphonon_b200.h")
MODULE = os.path.join(HERE, "fourphonon_b200.f90")

# Pointer arguments through which a call returns one scalar (not an array).
SCALAR_OUT = {
    "fp4_last_stats": {"n_processes", "n_contracted", "call_ms", "kernel_ms", "launches"},
    "fp4_server_admit": {"slot"},
    "fp4_server_tick": {"nfinished"},
    "fp4_server_collect": {"n_processes"},
    "fp4_server_status": {"running", "done", "bytes_in_use", "last_tick_ms", "ticks"},
}
# Entry points whose array arguments are device pointers.
DEVICE_POINTERS = {"fp4_np_driver_4ph_noalloc"}
COMPLEX = {"eigenvect"}

KIND = {"double": "real(c_double)", "float": "real(c_float)", "int": "integer(c_int)",
        "int32_t": "integer(c_int32_t)", "int64_t": "integer(c_int64_t)", "uint64_t": "integer(c_int64_t)",
        "uint16_t": "integer(c_int16_t)"}
HANDLES = {"fp4_ctx", "fp4_server", "void"}


def prototypes(src: str):
    """(return type, name, [(type text, argument name, array extent or None)])."""
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = []
    for m in re.finditer(r"\n([a-z_0-9 ]+?\**)\s*(fp4_\w+)\s*\(([^;]*?)\)\s*;", src):
        ret, name, args = " ".join(m.group(1).split()), m.group(2), m.group(3)
        params = []
        for a in args.split(","):
            a = " ".join(a.split())
            p = re.match(r"(.*?)(\w+)(?:\[(\d+)\])?$", a)
            params.append((p.group(1).strip(), p.group(2), int(p.group(3)) if p.group(3) else None))
        out.append((ret, name, params))
    return out


def constants(src: str):
    return [(m.group(1), int(m.group(2))) for m in re.finditer(r"#define (FP4_\w+) \(?(-?\d+)\)?", src)]


def dummy(fn: str, ctype: str, name: str, extent):
    """Declaration line of one dummy argument."""
    const = ctype.startswith("const ")
    base = ctype.replace("const ", "").replace("*", "").strip()
    stars = ctype.count("*")
    if base in HANDLES:
        if stars == 2:
            return f"type(c_ptr), intent(out) :: {name}"
        return f"type(c_ptr), value :: {name}"
    if base == "fp4_globals":
        return f"type(fp4_globals), intent(in) :: {name}"
    kind = KIND[base]
    if name in COMPLEX and base == "double":
        kind = "complex(c_double_complex)"
    if stars == 0 and extent is None:
        return f"{kind}, value :: {name}"
    if fn in DEVICE_POINTERS:
        return f"type(c_ptr), value :: {name}"
    intent = "intent(in)" if const else ("intent(out)" if name in SCALAR_OUT.get(fn, ()) else "intent(inout)")
    if name in SCALAR_OUT.get(fn, ()):
        return f"{kind}, {intent} :: {name}"
    return f"{kind}, {intent} :: {name}({extent if extent else '*'})"


def wrap(head: str, names, tail: str, indent: str):
    """head(names...) tail, continued with & so that no line passes 100 columns
    (free-form Fortran allows 132)."""
    lines, cur = [], head + "("
    for i, n in enumerate(names):
        piece = n + (", " if i + 1 < len(names) else "")
        if len(cur) + len(piece) > 100:
            lines.append(cur.rstrip() + " &")
            cur = indent + "     "
        cur += piece
    if len(cur) + 2 + len(tail) > 100:
        lines.append(cur + ") &")
        lines.append(indent + "     " + tail)
    else:
        lines.append(cur + ") " + tail)
    return lines


def render(src: str) -> str:
    L = ["! Generated by include/make_fortran_module.py from include/fourphonon_b200.h: do not edit.",
         "! ISO_C_BINDING interfaces of the B200 scattering-rate path.  Each function replaces the",
         "! Fortran subroutine named in the header's comment above its prototype and takes that",
         "! subroutine's arguments, in the same order, plus the context and the fp4_globals record.",
         "module fp4_b200",
         "  use iso_c_binding",
         "  implicit none",
         ""]
    for name, value in constants(src):
        L.append(f"  integer(c_int), parameter :: {name} = {value}")
    L += ["",
          "  ! The reference's module globals (Src/config.f90:9-47), fields in the header's order.",
          "  type, bind(c) :: fp4_globals",
          "     integer(c_int32_t) :: ngrid(3)",
          "     integer(c_int32_t) :: nbands",
          "     real(c_double)     :: rlattvec(3,3)",
          "     real(c_double)     :: T",
          "     real(c_double)     :: scalebroad",
          "     real(c_double)     :: omega_max",
          "     integer(c_int32_t) :: onlyharmonic",
          "     integer(c_int32_t) :: nelements",
          "     integer(c_int32_t) :: natoms",
          "     type(c_ptr)        :: masses",
          "     type(c_ptr)        :: types",
          "  end type fp4_globals",
          "",
          "  interface"]
    for ret, name, params in prototypes(src):
        rkind = {"int": "integer(c_int)", "int64_t": "integer(c_int64_t)", "const char *": "type(c_ptr)"}[ret]
        names = [p[1] for p in params]
        L += wrap(f"     {rkind} function {name}", names, f'bind(c, name="{name}")', "     ")
        L.append("       import :: c_ptr, c_int, c_int16_t, c_int32_t, c_int64_t, c_float, c_double, &")
        L.append("            c_double_complex, fp4_globals")
        for ctype, pname, extent in params:
            L.append("       " + dummy(name, ctype, pname, extent))
        L.append(f"     end function {name}")
        L.append("")
    L[-1:] = ["  end interface", "end module fp4_b200", ""]
    return "\n".join(L)


def main(argv):
    text = render(open(HEADER).read())
    if "--check" in argv:
        cur = open(MODULE).read() if os.path.exists(MODULE) else ""
        if cur != text:
            print(f"{MODULE} is stale: run python include/make_fortran_module.py", file=sys.stderr)
            return 1
        return 0
    with open(MODULE, "w") as f:
        f.write(text)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
