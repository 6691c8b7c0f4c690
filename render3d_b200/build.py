"""Builds libr3d_b200.so (sm_100a CUDA kernels + C-ABI + C23 host code) and
the r3d_headless command-line tool in place, next to this file.

    python render3d_b200/build.py [--force] [--verbose]

(run as a script: importing the package loads the library it builds)

Kernels are compiled with -fmad=false and IEEE division / square root: the
raycast's arithmetic is written out operation by operation (explicit fmaf)
and must not be contracted or approximated, so that the CPU oracle used by
the tests reproduces it bit for bit.  ptxas register / spill reports go to
_build/ptxas.log.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libr3d_b200.so")
CLI = os.path.join(HERE, "r3d_headless")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
# R3D_NVCC_EXTRA: extra nvcc flags (tuning experiments)
NVCC_FLAGS = GENCODE + os.environ.get("R3D_NVCC_EXTRA", "").split() + [
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xptxas", "-v", "-I" + INC, "-I" + CSRC,
]
# the image's CC points at a gcc build without libgomp; the system gcc is used
CC = shutil.which("gcc", path="/usr/bin:/bin") or "gcc"
C_FLAGS = ["-O2", "-std=c2x", "-D_GNU_SOURCE", "-fPIC", "-ffp-contract=off", "-Wall",
           "-Wextra", "-I" + INC, "-I" + os.path.join(CUDA_HOME, "include")]

CU_SOURCES = ["r3d_ctx.cu", "r3d_fwd.cu", "r3d_persist.cu", "r3d_noalloc.cu", "r3d_diff.cu",
              "r3d_batch.cu", "r3d_phantom.cu", "r3d_diag.cu", "r3d_shard.cu", "r3d_overlay.cu",
              "r3d_stream.cu", "r3d_slab.cu", "r3d_clip.cu", "r3d_vslab.cu", "r3d_surf.cu",
              "r3d_postfilter.cu", "r3d_staged.cu"]
# sources compiled once more per sampling path (-DR3D_FWD_PATH=p), so the
# paths' raycast kernels compile in parallel
PER_PATH = {"r3d_fwd.cu", "r3d_persist.cu"}
N_PATHS = 6
C_SOURCES = ["r3d_render.c", "r3d_host.c"]
CLI_SOURCES = ["r3d_headless.c"]


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _headers() -> list[str]:
    hs = []
    for d in (CSRC, INC):
        hs += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".h", ".cuh"))]
    return hs


def _run(cmd: list[str], log=None, verbose=False) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if log is not None:
        log.write(" ".join(cmd) + "\n" + r.stdout + "\n")
    if r.returncode != 0:
        sys.stderr.write(r.stdout)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]))


def _compile_jobs() -> list[tuple[list[str], str, str]]:
    """(compiler command without -c/-o, source, object) of every object."""
    jobs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        jobs.append(([NVCC] + NVCC_FLAGS, s, os.path.join(BUILD, src + ".o")))
        if src in PER_PATH:
            for p in range(N_PATHS):
                jobs.append(([NVCC] + NVCC_FLAGS + [f"-DR3D_FWD_PATH={p}"], s,
                             os.path.join(BUILD, f"{src}.p{p}.o")))
    for src in C_SOURCES:
        jobs.append(([CC] + C_FLAGS, os.path.join(CSRC, src), os.path.join(BUILD, src + ".o")))
    return jobs


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles whatever is out of date, in parallel; returns the library path."""
    import concurrent.futures as cf
    import io
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    jobs = _compile_jobs()
    objs = [o for _, _, o in jobs]
    todo = [(cmd, s, o) for cmd, s, o in jobs if force or _newer(o, [s] + hdrs)]
    with open(os.path.join(BUILD, "ptxas.log"), "a") as log:
        def one(job):
            cmd, s, o = job
            buf = io.StringIO()
            try:
                _run(cmd + ["-c", s, "-o", o], buf, verbose)
            finally:
                log.write(buf.getvalue())
        with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
            for f in [ex.submit(one, j) for j in todo]:
                f.result()
        if force or _newer(LIB, objs):
            _run([NVCC] + GENCODE + ["-shared", "-o", LIB] + objs +
                 ["-lcudart", "-lpthread", "-lm"], log, verbose)
        cli_src = [os.path.join(CSRC, s) for s in CLI_SOURCES]
        if force or _newer(CLI, cli_src + [LIB] + hdrs):
            _run([CC] + C_FLAGS + ["-o", CLI] + cli_src +
                 ["-L" + HERE, "-lr3d_b200", "-Wl,-rpath,$ORIGIN", "-lm"], log, verbose)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))


if __name__ == "__main__":
    main()
