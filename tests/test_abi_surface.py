"""CPU checks of the C-ABI library: it loads without a GPU, exports every
function include/*.h declares, and its struct layouts are the reference's."""
import ctypes
import os
import re

import numpy as np

from h261enc_cuda_b200 import _lib, compat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(h261\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_loads_and_exports_abi():
    lib = _lib.core()
    for name in _lib.ABI_SYMBOLS:
        assert hasattr(lib, name), name
    assert lib.h261b_version().startswith(b"h261b")


def test_every_declared_function_is_exported():
    lib = _lib.core()
    declared = _declared("h261b_abi.h") + _declared("h261b.h")
    assert len(declared) >= 16 + 15
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    synth = _lib.synth()
    for n in _declared("h261b_synth.h"):
        assert hasattr(synth, n), n


def test_abi_symbols_match_reference_header_list():
    abi = _declared("h261b_abi.h")
    assert sorted(_lib.ABI_SYMBOLS) == abi


def test_struct_layouts():
    assert ctypes.sizeof(compat.MeGpu) == 88
    assert ctypes.sizeof(compat.Macroblocks) == 208
    assert ctypes.sizeof(compat.Context) == 248
    assert _lib.MB_DTYPE.itemsize == 1572 and _lib.MB_DTYPE.fields["tcoeff"][1] == 28
    assert _lib.ME_MB_DTYPE.itemsize == 20


def test_session_bytes_and_no_device_errors():
    lib = _lib.core()
    qcif = lib.h261b_session_bytes(176, 144)
    cif = lib.h261b_session_bytes(352, 288)
    assert 2 * 38016 <= qcif < 2 * 38016 + 4096 and 2 * 152064 <= cif < 2 * 152064 + 4096
    assert lib.h261b_session_bytes(177, 144) < 0


def test_result_to_abi_expansion():
    """Compact results expand to the reference's macroblock records."""
    from h261enc_cuda_b200.engine import FrameResult
    mbs = np.zeros(2, _lib.RESULT_DTYPE)
    mbs["type"] = [0, 2]
    mbs["flags"] = [4, 7]
    mbs["quant"] = 8
    mbs["cbp"] = [63, 33]
    mbs["mvx"] = [0, -3]
    mbs["mvy"] = [0, 5]
    lv = np.zeros((2, 6, 64), np.int8)
    lv[0, :, 0] = np.array([200, 255, 1, 128, 17, 254], np.uint8).view(np.int8)
    lv[1, 0, 5 * 8 + 2] = -7          # column u = 5, row v = 2
    out = FrameResult(0, 0, 8, mbs, lv).to_abi(32)
    assert list(out["tcoeff"][0, :, 0]) == [200, 255, 1, 128, 17, 254]
    assert out["tcoeff"][1, 0, 2 * 8 + 5] == -7 and out["mv"][1].tolist() == [-3, 5]
    assert out["mb_x"].tolist() == [0, 16] and out["cbp"].tolist() == [63, 33]
