"""Build the C/OpenMP oracle (oracle/csrc/simp_cpu.c) into oracle/_build/.

Test and baseline infrastructure only. Generic x86-64-v3 code (AVX2/FMA) so
the library built in one container also runs on the GPU hosts' CPUs.
"""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "csrc" / "simp_cpu.c"
OUT = HERE / "_build" / "libsimp_cpu.so"


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("no C compiler found")
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".tmp.so")
    subprocess.run([cc, "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared",
                    "-o", str(tmp), str(SRC), "-lm"], check=True)
    tmp.replace(OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
