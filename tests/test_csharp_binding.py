"""The C# binding beside the header (include/GridSimB200.cs), checked without a .NET toolchain: every entry point of
the header has exactly one P/Invoke declaration whose return and parameter types match the C prototype, every
structure has the C layout field for field (sequential layout on x64, through the ctypes mirrors that
test_abi.py checks against the compiler's offsetof), and every constant equals the header's."""
import ctypes
import os
import re

import pytest

from gridsim_b200 import _abi
from tests.conftest import ROOT

HEADER = os.path.join(ROOT, "include", "gridsim_b200.h")
BINDING = os.path.join(ROOT, "include", "GridSimB200.cs")

CS_SCALARS = {"byte": (1, 1), "short": (2, 2), "int": (4, 4), "uint": (4, 4), "long": (8, 8), "ulong": (8, 8),
              "float": (4, 4), "double": (8, 8), "IntPtr": (8, 8), "UIntPtr": (8, 8)}
CTYPES_OF = {"int": (ctypes.c_int32,), "long": (ctypes.c_int64,), "ulong": (ctypes.c_uint64,),
             "double": (ctypes.c_double,), "IntPtr": (ctypes.c_void_p, ctypes.c_char_p)}


def _strip_cs_comments(text):
    return re.sub(r"//[^\n]*", "", text)


def _block(text, start):
    """The text between the brace that follows `start` and its match."""
    i = text.index("{", text.index(start))
    depth = 0
    for j in range(i, len(text)):
        depth += {"{": 1, "}": -1}.get(text[j], 0)
        if depth == 0:
            return text[i + 1:j]
    raise AssertionError(f"unbalanced braces after {start!r}")


def native_class():
    return _block(_strip_cs_comments(open(BINDING).read()), "static unsafe class GsNative")


def cs_structs():
    """C# struct name -> [(field, type, fixed count or None)] in declaration order."""
    out = {}
    body = native_class()
    for m in re.finditer(r"\[StructLayout\(LayoutKind\.Sequential\)\]\s*public struct (\w+)\s*\{(.*?)\}", body, re.S):
        fields = []
        for decl in m.group(2).split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            fm = re.fullmatch(r"public (fixed )?(\w+) (.+)", decl)
            assert fm, f"{m.group(1)}: unparsed field declaration {decl!r}"
            for name in fm.group(3).split(","):
                name = name.strip()
                if fm.group(1):
                    am = re.fullmatch(r"(\w+)\[(\d+)\]", name)
                    fields.append((am.group(1), fm.group(2), int(am.group(2))))
                else:
                    fields.append((name, fm.group(2), None))
        out[m.group(1)] = fields
    return out


def cs_layout(structs, name):
    """[(field, offset, size)], total size and alignment of a sequential struct on x64."""
    off, align, rows = 0, 1, []
    for fname, ftype, count in structs[name]:
        if ftype in CS_SCALARS:
            size, al = CS_SCALARS[ftype]
        else:
            _, size, al = cs_layout(structs, ftype)
        if count is not None:
            size *= count
        off = (off + al - 1) // al * al
        rows.append((fname, off, size))
        off += size
        align = max(align, al)
    return rows, (off + align - 1) // align * align, align


def c_name(cs_struct):
    return "gs_" + re.sub(r"(?<!^)(?=[A-Z])", "_", cs_struct).lower()


def header_text():
    return re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)


def header_prototypes():
    """name -> (return type, [(base type, pointer depth)])."""
    out = {}
    for m in re.finditer(r"(int|void|const\s+char\s*\*)\s*(gs_\w+)\s*\(([^)]*)\)\s*;", header_text()):
        params = []
        for p in m.group(3).split(","):
            p = p.strip()
            if p in ("", "void"):
                continue
            stars = p.count("*")
            words = [w for w in re.sub(r"\*", " ", p).split() if w != "const"]
            params.append((words[0], stars))
        ret = "const char *" if "char" in m.group(1) else m.group(1)
        out[m.group(2)] = (ret, params)
    return out


def cs_imports():
    """name -> (return type, [(attribute, modifier, type)])."""
    out = {}
    body = native_class()
    for m in re.finditer(r"\[DllImport\(Lib\)\]\s*public static extern ([\w\[\]?]+) (gs_\w+)\((.*?)\);", body, re.S):
        params = []
        for p in " ".join(m.group(3).split()).split(","):
            p = p.strip()
            if not p:
                continue
            pm = re.fullmatch(r"(\[\w+\] )?((?:ref|out|in) )?([\w\[\]?]+) \w+", p)
            assert pm, f"{m.group(2)}: unparsed parameter {p!r}"
            params.append(((pm.group(1) or "").strip(), (pm.group(2) or "").strip(), pm.group(3).rstrip("?")))
        assert m.group(2) not in out, f"{m.group(2)} is declared twice"
        out[m.group(2)] = (m.group(1), params)
    return out


def test_every_entry_point_is_declared_once():
    declared = set(header_prototypes())
    assert declared == set(_abi.EXPORTS), "the header scan and the ctypes table disagree"
    assert set(cs_imports()) == declared


def _param_matches(cs, c, structs):
    attr, mod, ty = cs
    base, stars = c
    ints = ("int", "int32_t")
    if mod in ("ref", "out", "in"):
        if ty in structs:
            return base == c_name(ty) and stars == 1
        if ty == "IntPtr":
            return stars == 2 and base.startswith("gs_")
        if ty == "int":
            return base in ints and stars == 1
        return False
    if ty.endswith("[]"):
        el = ty[:-2]
        if el == "IntPtr":
            return stars == 2 and base.startswith("gs_")
        if el in structs:
            return base == c_name(el) and stars == 1
        want = {"int": ints, "double": ("double",), "byte": ("uint8_t", "char"), "ulong": ("uint64_t",)}[el]
        return base in want and stars == 1
    if ty == "IntPtr":
        return stars == 1
    want = {"int": ints, "long": ("int64_t",), "double": ("double",), "UIntPtr": ("size_t",)}[ty]
    return base in want and stars == 0


def test_pinvoke_signatures_match_the_prototypes():
    structs = cs_structs()
    protos = header_prototypes()
    for name, (ret, params) in cs_imports().items():
        cret, cparams = protos[name]
        assert {"int": "int", "void": "void", "IntPtr": "const char *"}[ret] == cret, name
        assert len(params) == len(cparams), f"{name}: {len(params)} parameters, the header has {len(cparams)}"
        for k, (cs, c) in enumerate(zip(params, cparams)):
            assert _param_matches(cs, c, structs), f"{name} parameter {k}: C# {cs} against C {c}"
        # an array the library writes into is passed [Out] where the marshaller would otherwise copy it back
        # only for blittable types; struct arrays the library fills need the attribute
        for attr, mod, ty in params:
            if ty.endswith("[]") and ty[:-2] in structs and name == "gs_serve_poll":
                assert attr == "[Out]", f"{name}: {ty} is filled by the library"


@pytest.mark.parametrize("name", ["CtxOpts", "GridDesc", "PfOpts", "PfResult", "N1Result", "GridInfo", "MultiStats",
                                  "ServeOpts", "Request", "Response", "ServeStats", "Schedule"])
def test_struct_layouts_match_the_c_structs(name):
    structs = cs_structs()
    assert name in structs
    rows, size, _ = cs_layout(structs, name)
    cls = getattr(_abi, name)
    assert size == ctypes.sizeof(cls), f"{name}: C# size {size}, C size {ctypes.sizeof(cls)}"
    cfields = cls._fields_
    assert len(rows) == len(cfields), f"{name}: {len(rows)} fields, C has {len(cfields)}"
    for (fname, off, fsize), (cf, ct), (_, cty, count) in zip(rows, cfields, structs[name]):
        desc = getattr(cls, cf)
        assert (off, fsize) == (desc.offset, desc.size), f"{name}.{fname} against {cf}"
        if count is not None:
            assert issubclass(ct, ctypes.Array) and ct._length_ == count and ct._type_ is ctypes.c_int32, f"{name}.{fname}"
        elif cty in structs:
            assert ct is getattr(_abi, cty), f"{name}.{fname}"
        elif cty == "IntPtr":
            assert ct in CTYPES_OF["IntPtr"] or issubclass(ct, ctypes._Pointer), f"{name}.{fname}"
        else:
            assert ct in CTYPES_OF[cty], f"{name}.{fname}: C# {cty}, ctypes {ct}"


def test_every_struct_of_the_header_has_a_binding():
    c_structs = set(re.findall(r"typedef struct (gs_\w+) \{", header_text()))
    assert c_structs == {c_name(s) for s in cs_structs()}


def test_constants_equal_the_header():
    text = header_text()
    header = {}
    for body in re.findall(r"enum \w+ \{(.*?)\};", text, re.S):
        for k, v in re.findall(r"(GS_\w+)\s*=\s*(\d+)", body):
            header[k] = int(v)
    for k, v in re.findall(r"#define (GS_\w+) (\d+)", text):
        header[k] = int(v)
    cs = {}
    for decl in re.findall(r"public const int (.*?);", native_class(), re.S):
        for k, v in re.findall(r"(GS_\w+)\s*=\s*(\d+)", decl):
            cs[k] = int(v)
    assert cs == header


def test_binding_source_is_balanced():
    text = _strip_cs_comments(open(BINDING).read())
    text = re.sub(r'\$?"(?:[^"\\]|\\.)*"', '""', text)
    for o, c in ("{}", "()", "[]"):
        assert text.count(o) == text.count(c), f"unbalanced {o}{c}"
