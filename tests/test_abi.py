"""The C-ABI library loads and exports exactly what include/*.h declares.

No GPU is needed: only symbol lookup, no compute call.
"""
import glob
import os
import re
import subprocess

from conftest import ROOT
from disco2_b200 import lib

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*\**\s*\**(dgpu_[A-Za-z0-9_]+)\s*\(", re.M)


def declared_symbols() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(DECL.findall(text))
    return names


def exported_symbols() -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_library_loads_and_exports_every_declared_symbol():
    L = lib.load()
    decl = declared_symbols()
    assert len(decl) >= 25
    for name in sorted(decl):
        assert hasattr(L, name), name


def test_exports_are_exactly_the_declared_abi():
    exported = {s for s in exported_symbols() if not s.startswith("_")}
    assert exported == declared_symbols()


def test_python_binding_covers_the_header():
    assert set(lib.SIGNATURES) == declared_symbols()
