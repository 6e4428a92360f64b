"""Build libpolar.so (sm_100a) in-tree with nvcc.

    python -m polar_b200.csrc.build [--debug]

Compiles every .cu file in this directory into polar_b200/libpolar.so.  Also used by
__graft_entry__.build().
"""
import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
INCLUDE = ROOT / "include"
OUT = PKG / "libpolar.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    p = shutil.which("nvcc")
    if p:
        return p
    cand = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(HERE.glob("*.cu"))


def build(debug=False, verbose=False, out=OUT, extra=()):
    nvcc = nvcc_path()
    objdir = ROOT / "_build"
    objdir.mkdir(exist_ok=True)
    flags = ARCH + ["-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(INCLUDE), "-I", str(HERE),
                    "--expt-relaxed-constexpr"]
    flags += ["-O0", "-G"] if debug else ["-O3"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    flags += list(extra)
    objs = []
    procs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        objs.append(obj)
        cmd = [nvcc, "-c", str(src), "-o", str(obj)] + flags
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    ok = True
    for cmd, pr in procs:
        out_txt = pr.communicate()[0].decode()
        if pr.returncode != 0 or verbose:
            sys.stderr.write(out_txt)
        if pr.returncode != 0:
            sys.stderr.write("FAILED: " + " ".join(cmd) + "\n")
            ok = False
    if not ok:
        raise RuntimeError("nvcc compilation failed")
    tmp = Path(str(out) + ".tmp")
    link = [nvcc, "-shared", "-o", str(tmp)] + [str(o) for o in objs] + ARCH + ["-cudart", "static",
                                                                                "-Xlinker", "--no-undefined"]
    subprocess.check_call(link)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(debug=a.debug, verbose=a.verbose))
