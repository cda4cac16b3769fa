"""Build libcm_b200.so in-tree with nvcc for sm_100a.

    python -m contactmechanics_b200.build [--force] [--ptxas-verbose]
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "lib", "libcm_b200.so")
SOURCES = ["cm_plan.cu", "cm_op_p2.cu", "cm_batch.cu"]  # compiled in parallel
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + \
        [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, ptxas_verbose=False):
    if not force and not _stale():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    objdir = os.path.join(os.path.dirname(OUT), "obj")
    os.makedirs(objdir, exist_ok=True)
    base = [_nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE]
    if ptxas_verbose:
        base.append("-Xptxas=-v")
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(obj)
        procs.append(subprocess.Popen(base + ["-c", os.path.join(CSRC, src), "-o", obj],
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    failed = False
    for src, proc in zip(SOURCES, procs):
        out, err = proc.communicate()
        if proc.returncode != 0:
            sys.stderr.write(out + err)
            failed = True
        elif ptxas_verbose:
            sys.stdout.write(err)
    if failed:
        raise RuntimeError("nvcc failed building libcm_b200.so")
    link = [_nvcc(), *ARCH, "-shared", "-o", OUT + ".tmp"] + objs
    proc = subprocess.run(link, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed linking libcm_b200.so")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="--ptxas-verbose" in sys.argv)
    print(OUT)
