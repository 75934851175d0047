"""Build the engine's shared library in-tree for sm_100a:

    blind-spiking-lstm_b200/tfhe_b200/libtfhe_b200.so

nvcc compiles core.cu and one br_inst.cu and one br_inst64.cu object per
GLWE degree (log2 N = 7..12) in parallel, then links them with -shared.  The build is skipped when
the library is newer than every source.  Usage:

    python blind-spiking-lstm_b200/build.py [--force] [--jobs J]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OUT_DIR = os.path.join(HERE, "tfhe_b200")
LIB = os.path.join(OUT_DIR, "libtfhe_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")
LOGNS = (7, 8, 9, 10, 11, 12)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
                "-Xcompiler", "-O3", "-I" + INCLUDE, "-I" + CSRC]


def nvcc():
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the engine needs the CUDA toolkit to build")
    return path


def sources():
    out = []
    for name in sorted(os.listdir(CSRC)):
        if name.endswith((".cu", ".cuh", ".h")):
            out.append(os.path.join(CSRC, name))
    out.append(os.path.join(INCLUDE, "tfhe_b200.h"))
    return out


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources() + [__file__])


def _run(cmd):
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if proc.returncode != 0:
        raise RuntimeError("command failed:\n" + " ".join(cmd) + "\n" + proc.stdout)
    return proc.stdout


def build(force=False, jobs=None, verbose=False, extra_flags=()):
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    cc = nvcc()
    jobs = jobs or min(8, os.cpu_count() or 1)
    units = [("core", os.path.join(CSRC, "core.cu"), []), ("lstm_ops", os.path.join(CSRC, "lstm_ops.cu"), []),
             ("ks_tc", os.path.join(CSRC, "ks_tc.cu"), []), ("torus64", os.path.join(CSRC, "torus64.cu"), []),
              ("br_fp32", os.path.join(CSRC, "br_fp32.cu"), [])]
    units += [(f"br_n{lg}", os.path.join(CSRC, "br_inst.cu"), [f"-DBR_LOGN={lg}"]) for lg in LOGNS]
    units += [(f"br64_n{lg}", os.path.join(CSRC, "br_inst64.cu"), [f"-DBR_LOGN={lg}"]) for lg in LOGNS]
    cmds = []
    objs = []
    for name, src, defs in units:
        obj = os.path.join(OBJ_DIR, name + ".o")
        objs.append(obj)
        cmds.append([cc] + FLAGS + list(extra_flags) + defs + ["-c", src, "-o", obj])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for out in ex.map(_run, cmds):
            if verbose and out.strip():
                print(out)
    tmp = LIB + ".tmp"
    _run([cc] + ARCH + ["-shared", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-v", action="store_true", help="print register / shared-memory use")
    args = ap.parse_args()
    extra = ["-Xptxas", "-v"] if args.ptxas_v else []
    lib = build(force=args.force or args.ptxas_v, jobs=args.jobs, verbose=args.ptxas_v, extra_flags=extra)
    print(lib)


if __name__ == "__main__":
    sys.exit(main())
