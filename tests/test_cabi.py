"""The C-ABI library loads and exports every symbol include/neko_b200.h
declares (CPU only: no compute calls)."""
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    out = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if not name.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", name)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*\b((?:cuda|nb)_[a-z0-9_]+)\s*\(",
                             text, flags=re.M):
            out.add(m.group(1))
    return out


def test_header_symbols_exported(nblib):
    syms = declared_symbols()
    assert len(syms) > 25
    lib = os.path.join(ROOT, "neko_b200", "libnekob200.so")
    nm = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True,
                        check=True).stdout
    exported = {line.split()[-1] for line in nm.splitlines() if " T " in line}
    missing = sorted(syms - exported)
    assert not missing, missing
    for s in syms:
        getattr(nblib, s)  # resolvable through ctypes


def test_python_binding_covers_header():
    from neko_b200 import _lib
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_version(nblib):
    assert b"sm_100a" in nblib.nb_version()
