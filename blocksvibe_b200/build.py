"""Build libb3dgpu.so in place (sm_100a): one object per limb count plus the C ABI, compiled in parallel.

    python -m blocksvibe_b200.build [--force]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libb3dgpu.so")
BUILD = os.path.join(ROOT, "_build")
LIMBS = (6, 10, 14, 18, 22, 26, 30, 34, 38, 42, 46)
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _nvcc():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.isfile(p) or p == "nvcc"):
            return p
    raise RuntimeError("nvcc not found")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh", ".h", ".cpp"))] + \
           [os.path.join(ROOT, "include", "b3dgpu.h")]


def _stale():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(s) > t for s in _sources())


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(force=False, verbose=False):
    """compile every kernel for sm_100a and link blocksvibe_b200/libb3dgpu.so (skipped when up to date)"""
    if not force and not _stale():
        return OUT
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    jobs = [[nvcc, *ARCH, *FLAGS, f"-DB3D_L={L}", "-c", os.path.join(CSRC, "inst.cu"),
             "-o", os.path.join(BUILD, f"inst_L{L}.o")] for L in LIMBS]
    for unit in ("abi", "noalloc", "rns_mma", "json"):
        jobs.append([nvcc, *ARCH, *FLAGS, "-c", os.path.join(CSRC, f"{unit}.cu"), "-o", os.path.join(BUILD, f"{unit}.o")])
    for unit in ("plan", "setup_io"):                               # host C++ (the recursion's index plan)
        jobs.append([nvcc, *FLAGS, "-c", os.path.join(CSRC, f"{unit}.cpp"), "-o", os.path.join(BUILD, f"{unit}.o")])
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        for log in ex.map(_run, jobs):
            if verbose and log:
                print(log, file=sys.stderr)
    objs = [j[-1] for j in jobs]
    tmp = OUT + f".{os.getpid()}"
    _run([nvcc, *ARCH, "-shared", "-o", tmp, *objs])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
