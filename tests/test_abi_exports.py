"""The CUDA library loads without a GPU and exports every symbol include/wavefd_b200.h declares,
and the drop-in part of the header covers every export of the reference's libraries."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wavefd_b200.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", txt)) - {"if", "sizeof"})


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    return {l.split()[-1] for l in out.splitlines() if " T " in l}


@pytest.fixture(scope="module")
def libpath():
    from wavefd_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")
    return _lib.LIB_PATH


def test_library_loads_without_gpu(libpath):
    lib = ctypes.CDLL(libpath)
    assert hasattr(lib, "Prop3DAcoIsoDenQ_DEO2_FDTD_alloc")


def test_every_declared_symbol_is_exported(libpath):
    names = declared()
    assert len(names) > 150
    missing = [n for n in names if n not in exported(libpath)]
    assert not missing, missing


def test_reference_named_links(libpath):
    libdir = os.path.dirname(libpath)
    for n in ("prop2DAcoIsoDenQ_DEO2_FDTD", "prop2DAcoVTIDenQ_DEO2_FDTD", "prop2DAcoTTIDenQ_DEO2_FDTD",
              "prop3DAcoIsoDenQ_DEO2_FDTD", "prop3DAcoVTIDenQ_DEO2_FDTD", "prop3DAcoTTIDenQ_DEO2_FDTD", "spacetime"):
        p = os.path.join(libdir, f"lib{n}.so")
        assert os.path.exists(p), p


def test_header_covers_reference_exports(libpath):
    from oracle.oracle import REF_DIR
    strict = os.path.join(REF_DIR, "strict")
    if not os.path.isdir(strict):
        pytest.skip("reference not built")
    ours = exported(libpath)
    decl = set(declared())
    for f in sorted(os.listdir(strict)):
        if not f.startswith("libprop") and f != "libspacetime.so":
            continue
        ref = exported(os.path.join(strict, f))
        ref = {s for s in ref if s.startswith("Prop") or s.endswith("data_float") or s.endswith("data_double")}
        assert ref <= ours, (f, sorted(ref - ours))
        assert ref <= decl, (f, sorted(ref - decl))


# ---- signatures: the header's Part 1 prototypes against the reference's own definitions ----------
REF_SRC = os.environ.get("WAVEFD_REFERENCE_SRC") or os.path.join(os.path.dirname(ROOT), "reference", "src")


def _norm_type(decl):
    """ABI type of one parameter or return declaration: qualifiers that do not change the C ABI
    (const, __restrict__) dropped, the parameter name dropped, pointers attached to the type."""
    d = re.sub(r"\b(const|__restrict__|restrict)\b", " ", decl)
    d = re.sub(r"\s*\*\s*", " * ", d).split()
    if len(d) > 1 and re.match(r"^[A-Za-z_]\w*$", d[-1]) and d[-1] not in ("long", "float", "double", "int", "void",
                                                                           "size_t", "char"):
        d = d[:-1]  # parameter name
    return " ".join(d).replace(" *", "*")


def _prototypes(text, terminator):
    """name -> (return type, [parameter types]) of every top-level C function declared (';') or
    defined ('{') in text."""
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    out = {}
    pat = re.compile(r"(?:^|[;}\n])\s*((?:[A-Za-z_][\w]*[\s\*]+)+?)([A-Za-z_]\w*)\s*\(([^()]*)\)\s*" +
                     re.escape(terminator))
    for m in pat.finditer(text):
        ret, name, params = m.group(1), m.group(2), m.group(3)
        if ret.strip() in ("return", "else") or "extern" in ret and '"C"' in ret:
            continue
        ret = ret.replace('extern "C"', "")
        plist = [] if params.strip() in ("", "void") else [_norm_type(p) for p in params.split(",")]
        out[name] = (_norm_type(ret + " x"), plist)
    return out


def test_header_signatures_match_reference_definitions():
    if not os.path.isdir(REF_SRC):
        pytest.skip("reference sources not present")
    header = _prototypes(open(HEADER).read(), ";")
    checked = 0
    for f in sorted(os.listdir(REF_SRC)):
        if not (f.startswith("prop") and f.endswith(".cc")) and f != "spacetime.cc":
            continue
        ref = _prototypes(open(os.path.join(REF_SRC, f)).read(), "{")
        for name, sig in ref.items():
            if not (name.startswith("Prop") or name.endswith("data_float") or name.endswith("data_double")):
                continue
            assert name in header, f"{f}: {name} not declared in the header"
            assert header[name] == sig, f"{f}: {name}: header {header[name]} vs reference {sig}"
            checked += 1
    assert checked > 150, checked
