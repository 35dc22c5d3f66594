"""Compile the C oracle (test infrastructure / CPU baseline) with gcc + OpenMP.

    python -m oracle.build_oracle
"""
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "ppt_oracle.c"
LIB = HERE / "lib" / "libppt_oracle.so"


def build(force=False):
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("gcc not found: the C oracle needs a C compiler")
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [cc, "-O2", "-fopenmp", "-fPIC", "-shared", "-o", str(tmp), str(SRC), "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + res.stderr)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True))
