"""
Build the native library ``_native/libaimd_b200.so`` for sm_100a.

The class-templated kernels are split into one translation unit per bra pair
class (csrc/hf_class_jk.cu, -DAIMD_CLASS=0..5) and per (bra, ket) class pair
for the gradient (csrc/hf_class_grad.cu, -DAIMD_CLASS=X -DAIMD_KET=Y) plus the
one-electron unit and the C-ABI unit, compiled in parallel and linked with
the static CUDA runtime. Objects are rebuilt only when a source is newer.

    python -m aimd_b200.build      (or __graft_entry__.build())
"""

from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import time
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
CSRC = os.path.join(PKG_ROOT, "csrc")
INCLUDE = os.path.join(os.path.dirname(PKG_ROOT), "include")
OUT_DIR = os.path.join(HERE, "_native")
OBJ_DIR = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(OUT_DIR, "libaimd_b200.so")
# the device SCF driver: a second library over the first, cuBLAS and cuSOLVER
SCF_SRC = os.path.join(CSRC, "hf_scf.cu")
SCF_OBJ = os.path.join(OBJ_DIR, "hf_scf.o")
SCF_LIB = os.path.join(OUT_DIR, "libaimd_scf.so")

NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
         "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]


def _units() -> list[tuple[str, str, list[str]]]:
    # one unit per class (and ket class) and arithmetic type (0 FP64, 1 FP32)
    units = [(os.path.join(CSRC, "hf_class_jk.cu"), os.path.join(OBJ_DIR, f"hf_class_jk_{x}_r{r}.o"),
              [f"-DAIMD_CLASS={x}", f"-DAIMD_REAL={r}"]) for x in range(6) for r in (0, 1)]
    units += [(os.path.join(CSRC, "hf_class_grad.cu"), os.path.join(OBJ_DIR, f"hf_class_grad_{x}_{y}_r{r}.o"),
               [f"-DAIMD_CLASS={x}", f"-DAIMD_KET={y}", f"-DAIMD_REAL={r}"])
              for x in range(6) for y in range(x + 1) for r in (0, 1)]
    # slowest units first so the parallel build finishes sooner (a J/K unit
    # of class X takes about as long as the gradient units of (X, X))
    def cost(u):
        v = [int(f.split("=")[1]) for f in u[2]]
        return 2 * v[0] + 1 if "hf_class_jk" in u[0] else v[0] + v[1]
    units.sort(key=lambda u: -cost(u))
    units.append((os.path.join(CSRC, "hf_onee.cu"), os.path.join(OBJ_DIR, "hf_onee.o"), []))
    units.append((os.path.join(CSRC, "hf_kernels.cu"), os.path.join(OBJ_DIR, "hf_kernels.o"), []))
    return units


def _includes(path: str, seen: set[str]) -> set[str]:
    """The file and every file it includes with #include "..." (transitively)."""
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include") and '"' in line:
                inc = line.split('"')[1]
                for base in (os.path.dirname(path), CSRC, INCLUDE):
                    cand = os.path.join(base, inc)
                    if os.path.exists(cand):
                        _includes(cand, seen)
                        break
    return seen


def _newest_dependency(src: str) -> float:
    """Modification time of the newest file the unit compiles from (its source and its includes)."""
    return max(os.path.getmtime(f) for f in _includes(src, set()))


def _compile(unit, verbose: bool) -> str:
    src, obj, extra = unit
    cmd = [NVCC, *FLAGS, *extra, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(obj)}:\n{res.stderr[-4000:]}")
    return res.stderr


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    todo = [u for u in _units()
            if force or not os.path.exists(u[1]) or os.path.getmtime(u[1]) < _newest_dependency(u[0])]
    logs = []
    if todo:
        # objects are stamped with the time the build started, so a source
        # edited while they compile is newer than them and the next build
        # compiles them again
        start = time.time()

        def one(u):
            log = _compile(u, verbose)
            os.utime(u[1], (start, start))
            return log
        with cf.ThreadPoolExecutor(max_workers=jobs or min(len(todo), os.cpu_count() or 4)) as ex:
            logs = list(ex.map(one, todo))
    relinked = False
    if todo or not os.path.exists(LIB):
        objs = [u[1] for u in _units()]
        res = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
                              "-Xlinker", "-soname=libaimd_b200.so", "-o", LIB], capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
        relinked = True
    if os.path.exists(SCF_SRC):
        stale = force or not os.path.exists(SCF_OBJ) or os.path.getmtime(SCF_OBJ) < _newest_dependency(SCF_SRC)
        if stale:
            logs.append(_compile((SCF_SRC, SCF_OBJ, []), verbose))
        if stale or relinked or not os.path.exists(SCF_LIB):
            cuda_lib = os.path.join(os.path.dirname(os.path.dirname(shutil.which(NVCC) or NVCC)), "lib64")
            res = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", SCF_OBJ,
                                  "-L", OUT_DIR, "-laimd_b200", "-L", cuda_lib, "-lcublas", "-lcusolver",
                                  "-Xlinker", "-rpath=$ORIGIN", "-Xlinker", f"-rpath={cuda_lib}", "-o", SCF_LIB],
                                 capture_output=True, text=True)
            if res.returncode != 0:
                raise RuntimeError(f"link of the SCF driver failed:\n{res.stderr[-4000:]}")
    if verbose:
        for log in logs:
            sys.stderr.write(log)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
