"""The C-ABI library loads and exports exactly what include/*.h declares.

No GPU is needed: only symbol lookup, no compute call.
"""
import glob
import os
import re
import subprocess

import pytest

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


def test_binding_links_the_library_abi():
    """The compiled Disco2-side binding (oracle/binding) resolves its dgpu_*
    calls against libdisco_gpu.so."""
    import oracle
    if not os.path.exists(oracle.BINDING_BIN):
        pytest.skip("binding not built (needs the reference sources)")
    out = subprocess.run(["nm", "-D", "--undefined-only", oracle.BINDING_BIN], capture_output=True,
                         text=True, check=True).stdout
    used = {ln.split()[-1] for ln in out.splitlines() if "dgpu_" in ln}
    assert {"dgpu_create", "dgpu_set_state", "dgpu_step_rk2", "dgpu_get_state", "dgpu_set_fused"} <= used
    ldd = subprocess.run(["ldd", oracle.BINDING_BIN], capture_output=True, text=True).stdout
    assert "libdisco_gpu.so" in ldd and "not found" not in ldd
