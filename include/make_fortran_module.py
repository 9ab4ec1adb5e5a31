"""Writes include/lica_gpu.f90, the Fortran 2003 ISO_C_BINDING module of include/lica_gpu.h:
the status codes, a bind(c) derived type for each struct, and an interface for each entry
point, so a Fortran solver can `use lica_gpu` and call the library directly.

Mapping:
  int32_t / int64_t / uint64_t / size_t / double / float scalars -> value arguments;
  host arrays (functions without the _device suffix) -> assumed-size arrays by reference;
  every pointer of a _device entry point, void*, opaque handles -> type(c_ptr), value;
  handle outputs (T**) and arrays of pointers -> type(c_ptr) by reference;
  struct pointers -> the bind(c) derived type by reference;  char* -> character(c_char)(*).

Run from the repository root: python include/make_fortran_module.py
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(HERE, "lica_gpu.h")
OUT = os.path.join(HERE, "lica_gpu.f90")

SCALAR = {"double": "real(c_double)", "float": "real(c_float)", "int32_t": "integer(c_int32_t)",
          "int64_t": "integer(c_int64_t)", "uint64_t": "integer(c_int64_t)", "size_t": "integer(c_size_t)",
          "int": "integer(c_int)"}
RESULT = {"int": "integer(c_int)", "int64_t": "integer(c_int64_t)", "size_t": "integer(c_size_t)",
          "const char*": "type(c_ptr)"}
# pointer arguments of host entry points that are one value, not an array
SCALAR_OUT = {("lica_col_fld_dims", "n"), ("lica_mg_profile_read", "total_ms"), ("lica_mg_profile_read", "launches")}
# struct pointer arguments that are arrays of structs
STRUCT_ARRAYS = {("lica_gpu_column_batch_create", "props"), ("lica_mg_solve_host_batch", "res"),
                 ("lica_gpu_bubble_tracking", "out")}


def strip_comments(txt):
    return re.sub(r"/\*.*?\*/", "", txt, flags=re.S)


def parse(txt):
    txt = strip_comments(txt)
    enums = re.findall(r"\b(LICA_\w+)\s*=\s*(\d+)", txt)
    opaque = set(re.findall(r"typedef\s+struct\s+\w+\s+(\w+)\s*;", txt))
    structs = []
    for body, name in re.findall(r"typedef\s+struct\s*\{(.*?)\}\s*(\w+)\s*;", txt, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"(?:const\s+)?(\w+)\s*(.*)", decl)
            ctype, rest = m.group(1), m.group(2)
            for d in rest.split(","):
                d = d.strip()
                ptr = d.startswith("*")
                d = d.lstrip("* ").strip()
                dim = None
                am = re.match(r"(\w+)\s*\[(\d+)\]", d)
                if am:
                    d, dim = am.group(1), int(am.group(2))
                fields.append((d, "type(c_ptr)" if ptr else SCALAR[ctype], dim))
        structs.append((name, fields))
    funcs = []
    for m in re.finditer(r"\n(\w[\w\s\*]*?)\b(lica_\w+)\s*\(([^)]*)\)\s*;", txt):
        ret = " ".join(m.group(1).split()).replace(" *", "*")
        params = []
        ptxt = " ".join(m.group(3).split())
        if ptxt != "void":
            for p in ptxt.split(","):
                p = p.strip()
                name = re.findall(r"(\w+)\s*$", p)[0]
                ctype = p[: len(p) - len(name)].strip()
                params.append((name, ctype))
        funcs.append((m.group(2), ret, params))
    return enums, opaque, structs, funcs


def fortran_arg(func, name, ctype, opaque, structs):
    device = func.endswith("_device")
    is_const = ctype.startswith("const ")
    base = ctype.replace("const ", "").replace(" ", "")
    stars = base.count("*")
    base = base.replace("*", "")
    intent = "intent(in)" if is_const else "intent(inout)"
    if stars == 0:
        return f"{SCALAR[base]}, value :: {name}"
    if base in opaque:
        return f"type(c_ptr), intent(out) :: {name}" if stars == 2 else f"type(c_ptr), value :: {name}"
    if stars == 2:
        return f"type(c_ptr), intent(in) :: {name}(*)"
    if base in structs:
        suffix = "(*)" if (func, name) in STRUCT_ARRAYS else ""
        return f"type({base}), {intent} :: {name}{suffix}"
    if base == "void" or device:
        return f"type(c_ptr), value :: {name}"
    if base == "char":
        return f"character(kind=c_char), {intent} :: {name}(*)"
    if (func, name) in SCALAR_OUT:
        return f"{SCALAR[base]}, intent(out) :: {name}"
    return f"{SCALAR[base]}, {intent} :: {name}(*)"


def wrap(head, names, tail, indent):
    """A statement with an argument list, continued with & so no line passes 100 columns."""
    lines = []
    cur = indent + head + "("
    for i, n in enumerate(names):
        piece = n + (", " if i < len(names) - 1 else ")")
        if len(cur) + len(piece) > 96:
            lines.append(cur.rstrip() + " &")
            cur = indent + "    " + piece
        else:
            cur += piece
    if not names:
        cur += ")"
    if len(cur) + len(tail) + 1 > 96:
        lines.append(cur + " &")
        cur = indent + "    " + tail
    else:
        cur += " " + tail
    lines.append(cur)
    return lines


def generate():
    enums, opaque, structs, funcs = parse(open(HEADER).read())
    struct_names = {s for s, _ in structs}
    o = ["! lica_gpu.f90 -- Fortran 2003 ISO_C_BINDING interface to include/lica_gpu.h, written by",
         "! include/make_fortran_module.py from the header (do not edit by hand).  A Fortran solver",
         "! calls the library with `use lica_gpu`; opaque handles are type(c_ptr), device arrays",
         "! are passed as type(c_ptr) device addresses, host arrays by reference.",
         "module lica_gpu",
         "  use, intrinsic :: iso_c_binding",
         "  implicit none",
         ""]
    for name, val in enums:
        o.append(f"  integer(c_int), parameter :: {name} = {val}")
    o.append("")
    for name, fields in structs:
        o.append(f"  type, bind(c) :: {name}")
        for fname, ftype, dim in fields:
            o.append(f"    {ftype} :: {fname}" + (f"({dim})" if dim else ""))
        o.append(f"  end type {name}")
        o.append("")
    o.append("  interface")
    for fname, ret, params in funcs:
        names = [p for p, _ in params]
        o.extend(wrap(f"{RESULT[ret]} function {fname}", names, f'bind(c, name="{fname}")', "    "))
        o.append("      import")
        for pname, ctype in params:
            o.append("      " + fortran_arg(fname, pname, ctype, opaque, struct_names))
        o.append(f"    end function {fname}")
        o.append("")
    o[-1:] = ["  end interface", "end module lica_gpu", ""]
    return "\n".join(o)


if __name__ == "__main__":
    text = generate()
    if "--check" in sys.argv:
        sys.exit(0 if open(OUT).read() == text else 1)
    with open(OUT, "w") as f:
        f.write(text)
