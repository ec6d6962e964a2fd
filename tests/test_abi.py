"""The C-ABI library loads without a GPU and exports every declared symbol."""
import ctypes
import os
import re

import numpy as np
import pytest

import qpanda_b200
from qpanda_b200.capi import GATE_DTYPE, LIB_PATH

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


EMU_HDR = "qpanda_b200_gpuemu.h"
EMU_LIB = os.path.join(os.path.dirname(LIB_PATH), "libGPUEmulator.so")


def declared():
    names = set()
    for f in os.listdir(HDR):
        if f.endswith(".h") and f != EMU_HDR:
            txt = open(os.path.join(HDR, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(qs\w+)\s*\(", txt, flags=re.M))
    return sorted(names)


def declared_emu():
    """Every function of the GPU-emulator plug-in header (gate names of the
    reference's GPUGatesDecl.h plus the two qs_gpuemu_* calls)."""
    txt = open(os.path.join(HDR, EMU_HDR)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = set(re.findall(r"^(?:bool|int|void)\s+(\w+)\s*\(", txt, flags=re.M))
    # C++ names bound to another exported symbol with an assembler label
    for cxx, sym in re.findall(r"^(?:bool|int|void)\s+(\w+)\s*\([^;]*?__asm__\(\"(\w+)\"\)", txt, flags=re.M | re.S):
        names.discard(cxx)
        names.add(sym)
    return sorted(names)


def test_emulator_header_lists_the_reference_names():
    names = declared_emu()
    for n in ("initstate", "clearState", "Hadamard", "RXdagger", "qubitmeasure", "controlRZdagger",
              "toffoli", "qbReset", "pMeasurenew", "getState", "pCRdagger"):
        assert n in names


@pytest.mark.parametrize("name", declared_emu())
def test_emulator_symbol_exported(name):
    L = ctypes.CDLL(EMU_LIB)
    assert hasattr(L, name), f"{name} declared in {EMU_HDR} but not exported by libGPUEmulator.so"


def test_library_exists_and_loads():
    assert os.path.exists(LIB_PATH)
    L = qpanda_b200.lib()
    assert b"sm_100a" in L.qs_version()


@pytest.mark.parametrize("name", declared())
def test_symbol_exported(name):
    L = ctypes.CDLL(LIB_PATH)
    assert hasattr(L, name), f"{name} declared in include/ but not exported"


def test_gate_record_layout():
    assert GATE_DTYPE.itemsize == 96
    assert GATE_DTYPE.fields["theta"][1] == 88
    assert GATE_DTYPE.fields["ctrl"][1] == 24


def test_errors_without_device_are_loud():
    L = qpanda_b200.lib()
    h = ctypes.c_void_p()
    rc = L.qs_create(0, 0, None, ctypes.byref(h))
    assert rc == -1 and b"qubit count" in L.qs_last_error()
    rc = L.qs_create(4, 7, None, ctypes.byref(h))
    assert rc == -1
    assert L.qs_gate_apply(None, None) == -1
