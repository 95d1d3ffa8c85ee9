"""Build recipe of the oracle (CPU restatement of the reference path; test
infrastructure only):

    python oracle/build.py      # -> oracle/_build/liboracle.so

-O3 with OpenMP; the ISA level is x86-64-v3 (AVX2/FMA) so the library built
here also runs on the GPU hosts' CPUs.
"""
from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build" / "liboracle.so"


def build() -> Path:
    OUT.parent.mkdir(exist_ok=True)
    src = HERE / "oracle.cpp"
    if OUT.exists() and OUT.stat().st_mtime >= src.stat().st_mtime:
        return OUT
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-O3", "-march=x86-64-v3", "-fopenmp", "-std=c++17", "-shared", "-fPIC",
           str(src), "-o", str(OUT)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stderr}")
    return OUT


if __name__ == "__main__":
    print(build())
    sys.exit(0)
