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


def _newest_source() -> float:
    files = glob.glob(os.path.join(CSRC, "*")) + glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(f) for f in files)


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
    newest = _newest_source()
    todo = [u for u in _units() if force or not os.path.exists(u[1]) or os.path.getmtime(u[1]) < newest]
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
    if todo or not os.path.exists(LIB):
        objs = [u[1] for u in _units()]
        res = subprocess.run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", LIB],
                             capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr[-4000:]}")
    if verbose:
        for log in logs:
            sys.stderr.write(log)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
