"""Builds libgitmvert.so in-tree with nvcc for sm_100a.

    python -m gitm_b200.build          # incremental
    python -m gitm_b200.build --force
    python -m gitm_b200.build -v       # with ptxas register / spill reports

Every translation unit is compiled to an object in gitm_b200/_build (in
parallel), then the objects are linked into the shared library.  The step
kernel is compiled once per entry of GV_STEP_INSTANCES (csrc/vert_instances.h),
each in a unit of its own (csrc/vert_instance.cu with that entry's -D values).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgitmvert.so")
SOURCES = ["gitm_vert.cu", "vert_adjoint.cu", "hz_kernel.cu"]
DEPS = ["gitm_vert.cu", "vert_adjoint.cu", "hz_kernel.cu", "vert_instance.cu", "vert_instances.h", "vert_kernel.cuh",
        "vert_ausm.cuh", "vert_adjoint.cuh", "vert_common.cuh", "vert_hz.cuh"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def instances() -> list[tuple[str, list[str]]]:
    """(id, -D flags) of every GV_STEP_INSTANCES entry."""
    text = open(os.path.join(CSRC, "vert_instances.h")).read()
    body = text[text.index("#define GV_STEP_INSTANCES(X)"):].split("\n\n", 1)[0]
    out = []
    for m in re.finditer(r"X\((\w+),\s*(\d+),\s*(\d+),\s*(\d+),\s*(true|false),\s*(\d+),\s*(true|false),\s*(\d+),"
                         r"\s*(true|false)\)", body):
        gid, io, nt, minb, acc, solver, save, na, og = m.groups()
        out.append((gid, [f"-DGV_ID={gid}", f"-DGV_IO={io}", f"-DGV_NT={nt}", f"-DGV_MINB={minb}",
                          f"-DGV_ACC={acc}", f"-DGV_SOLVER={solver}", f"-DGV_SAVE={save}", f"-DGV_NA={na}",
                          f"-DGV_OG={og}"]))
    if not out:
        raise RuntimeError("no step-kernel instances found in vert_instances.h")
    return out


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, d) for d in DEPS]
    deps.append(os.path.join(HERE, "..", "include", "gitm_vert.h"))
    deps.append(os.path.join(HERE, "..", "include", "gitm_hz.h"))
    deps.append(os.path.abspath(__file__))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose else []
    jobs = [(os.path.join(CSRC, s), [], os.path.join(BUILD, s[:-3] + ".o")) for s in SOURCES]
    # the adjoint kernel for members of 50 altitudes, in a unit of its own
    jobs.append((os.path.join(CSRC, "vert_adjoint.cu"), ["-DGV_ADJ_NA=50"], os.path.join(BUILD, "vert_adjoint_n50.o")))
    jobs += [(os.path.join(CSRC, "vert_instance.cu"), flags, os.path.join(BUILD, f"step_{gid}.o"))
             for gid, flags in instances()]

    def compile_one(job):
        src, flags, obj = job
        cmd = [nvcc(), *NVCC_FLAGS, *extra, *flags, "-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return obj, r.returncode, r.stdout + r.stderr

    workers = max(1, min(len(jobs), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(workers) as ex:
        results = list(ex.map(compile_one, jobs))
    failed = False
    for obj, rc, log in results:
        if log.strip() and (verbose or rc):
            sys.stderr.write(f"== {os.path.basename(obj)}\n{log}")
        failed = failed or rc != 0
    if failed:
        raise RuntimeError("nvcc failed (messages above)")
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", *[obj for obj, _, _ in results], "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
