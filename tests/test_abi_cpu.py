"""The C-ABI library loads and exports every symbol include/tara2d_gpu.h
declares (no compute call; no GPU needed)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "tara2d_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = set(re.findall(r"\b([a-z_0-9]+)\s*\(", txt))
    names = {n for n in names if n not in ("if", "sizeof")}
    names |= set(re.findall(r"extern\s+double\s+([a-z_0-9]+)\s*\[", txt))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    for must in ("derive2coh_", "ab2coh_", "derive2com_", "ab2com_", "rk4_nk2coh_", "pc_uky2coh_",
                 "tara_open", "tara_step", "comm_", "derive3com_", "ab3com_", "tara3d_open", "tara3d_step"):
        assert must in names


def test_library_exports_every_declared_symbol(tara):
    lib = tara.lib()
    missing = []
    for n in declared_symbols():
        try:
            getattr(lib, n)
        except AttributeError:
            try:
                ctypes.c_double.in_dll(lib, n)
            except ValueError:
                missing.append(n)
    assert not missing, missing
