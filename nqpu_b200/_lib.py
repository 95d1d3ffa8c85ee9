"""ctypes binding of the engine's C ABI (include/nqpu_b200.h).

The prototypes are read from the header itself, so every declared entry point
is bound with its exact argument and return types.  Loading fails loudly when
the shared library is missing: there is no pure-Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

PKG = Path(__file__).resolve().parent
HEADER = PKG.parent / "include" / "nqpu_b200.h"
LIB_PATH = PKG / "libnqpu_b200.so"


class NqpuComplex(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class NqpuMeasurement(C.Structure):
    _fields_ = [("outcome", C.c_uint32), ("probability", C.c_double)]


class NqpuVersion(C.Structure):
    _fields_ = [("major", C.c_uint32), ("minor", C.c_uint32), ("patch", C.c_uint32)]


class NqpuServerConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("max_qubits", C.c_uint32), ("lanes", C.c_uint32),
                ("large_lanes", C.c_uint32), ("large_qubits", C.c_uint32), ("max_shots", C.c_uint32)]


_SCALARS = {
    "void": None,
    "bool": C.c_bool,
    "uint32_t": C.c_uint32,
    "uint64_t": C.c_uint64,
    "int": C.c_int,
    "double": C.c_double,
    "float": C.c_float,
    "NqpuError": C.c_int,
    "NqpuDtype": C.c_int,
    "NqpuMode": C.c_int,
    "NqpuBatchParam": C.c_int,
    "NqpuRequestKind": C.c_int,
    "NqpuOptLevel": C.c_int,
    "NqpuServerConfig": NqpuServerConfig,
    "int32_t": C.c_int32,
    "NqpuComplex": NqpuComplex,
    "NqpuVersion": NqpuVersion,
    "NqpuMeasurement": NqpuMeasurement,
}

_PROTO = re.compile(r"^\s*(?:const\s+)?([A-Za-z_][A-Za-z0-9_]*)\s*(\*?)\s*(nqpu_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", re.M)


def _ctype(decl: str):
    decl = decl.strip()
    if decl == "void" or decl == "":
        return None
    decl = re.sub(r"\bconst\b", "", decl).strip()
    ptr = decl.count("*")
    base = decl.replace("*", " ").split()[0]
    if ptr == 0:
        return _SCALARS[base]
    if base in ("NqpuState", "NqpuCircuit", "NqpuServer", "NqpuBatch") or base == "void":
        return C.c_void_p
    if base == "char":
        return C.c_char_p
    return C.POINTER(_SCALARS[base])


def parse_header(path: Path = HEADER) -> dict[str, tuple]:
    """Return {name: (restype, [argtypes])} for every nqpu_* prototype."""
    text = path.read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"\s*\n\s*", " ", text)  # join multi-line prototypes
    text = text.replace(";", ";\n")
    out = {}
    for m in _PROTO.finditer(text):
        ret_base, ret_ptr, name, args = m.groups()
        if ret_ptr:
            restype = C.c_char_p if ret_base == "char" else C.c_void_p
        else:
            restype = _SCALARS[ret_base]
        argtypes = []
        for a in [x for x in args.split(",") if x.strip() and x.strip() != "void"]:
            # drop the parameter name
            a = a.strip()
            a = re.sub(r"([A-Za-z_][A-Za-z0-9_]*)\s*$", "", a) if re.search(r"[\s*][A-Za-z_][A-Za-z0-9_]*\s*$", a) else a
            argtypes.append(_ctype(a))
        out[name] = (restype, argtypes)
    return out


_lib = None


def load(path: Path | str | None = None) -> C.CDLL:
    """Load the engine library (built in-tree by nqpu_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("NQPU_B200_LIB", LIB_PATH))
    if not p.exists():
        raise RuntimeError(f"nqpu_b200 native library not built: {p} (run python -m nqpu_b200.build)")
    lib = C.CDLL(str(p))
    for name, (restype, argtypes) in parse_header().items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _lib = lib
    return lib


ERRORS = {
    0: "NQPU_OK", 1: "NQPU_INVALID_QUBIT", 2: "NQPU_INVALID_PARAMETER", 3: "NQPU_ALLOCATION_FAILED",
    4: "NQPU_SIMULATION_FAILED", 5: "NQPU_NULL_POINTER", 6: "NQPU_INVALID_HANDLE",
}


class NqpuErrorException(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        super().__init__(f"{where}: {ERRORS.get(code, code)}")


def check(code: int, where: str = "") -> None:
    if code != 0:
        raise NqpuErrorException(code, where)
