"""Build the engine in-tree: CUDA sources for sm_100a with nvcc, the C host
driver with gcc, linked into esthera_b200/libesthera_b200.so (CUDA runtime
linked statically) plus the reference-style command line esthera_b200/pf_cli.

Incremental: an object is rebuilt when its source or any header is newer.
Usage: python -m esthera_b200.build [-j JOBS] [--force]
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
INCLUDE = ROOT / "include"
OBJ = ROOT / "_build" / "obj"
LIB = PKG / "libesthera_b200.so"
CLI = PKG / "pf_cli"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no implicit multiply-add contraction, so every kernel that
# inlines a model or a scan computes bit-identical results (the device code
# writes its multiply-adds as explicit fmaf where it wants them).
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "--fmad=false",
              "-I" + str(INCLUDE), "-I" + str(CSRC)] + ARCH
CC_FLAGS = ["-O2", "-fPIC", "-std=gnu11", "-Wall", "-I" + str(INCLUDE)]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _cc():
    return "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else (shutil.which("gcc") or "cc")


def _stale(obj, src, deps):
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(d.stat().st_mtime > t for d in deps)


def build(jobs=None, force=False, verbose=False):
    OBJ.mkdir(parents=True, exist_ok=True)
    nvcc, cc = _nvcc(), _cc()
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.inc")) + list(INCLUDE.glob("*.h"))
    tasks = []
    for src in sorted(CSRC.glob("*.cu")):
        obj = OBJ / (src.stem + ".o")
        if force or _stale(obj, src, headers):
            tasks.append([nvcc] + NVCC_FLAGS + ["-c", str(src), "-o", str(obj)])
    for src in sorted(HOST.glob("*.c")):
        if src.name == "pf_cli.c":
            continue
        obj = OBJ / (src.stem + ".o")
        if force or _stale(obj, src, list(INCLUDE.glob("*.h"))):
            tasks.append([cc] + CC_FLAGS + ["-c", str(src), "-o", str(obj)])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("build failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
        return cmd

    if tasks:
        with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(run, tasks))
    objs = [str(OBJ / (s.stem + ".o")) for s in sorted(CSRC.glob("*.cu"))]
    objs += [str(OBJ / (s.stem + ".o")) for s in sorted(HOST.glob("*.c")) if s.name != "pf_cli.c"]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        run([nvcc, "-shared"] + ARCH + ["-o", str(LIB)] + objs + ["-lm"])
    if force or not CLI.exists() or CLI.stat().st_mtime < LIB.stat().st_mtime:
        run([cc] + CC_FLAGS + [str(HOST / "pf_cli.c"), "-o", str(CLI), "-L" + str(PKG), "-lesthera_b200",
                               "-Wl,-rpath,$ORIGIN", "-lm"])
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.jobs, a.force, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
