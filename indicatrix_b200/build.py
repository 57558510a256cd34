"""Builds ``libix_cuda.so`` in-tree for sm_100a.

The transport and metrics units are compiled twice -- reference-exact rounding
(``-DIX_EXACT=1 -fmad=false``) and the fast build (``-DIX_EXACT=0``: contraction,
approximate divide / square root, denormal flushing) -- and linked with the C-ABI host
code into one shared library beside this file.
Run ``python -m indicatrix_b200.build`` or call :func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.normpath(os.path.join(HERE, "..", "include"))
OUT = os.path.join(HERE, "libix_cuda.so")
BUILD_DIR = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _cuda_home(nvcc: str) -> str:
    return os.path.dirname(os.path.dirname(os.path.realpath(nvcc)))


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [
        os.path.join(INCLUDE, f) for f in sorted(os.listdir(INCLUDE))
    ]


def _up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(s) <= t for s in _sources() + [__file__])


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the CUDA extension if any source is newer than the library."""
    if not force and _up_to_date():
        return OUT
    nvcc = _nvcc()
    os.makedirs(BUILD_DIR, exist_ok=True)
    common = [nvcc, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-Xptxas", "-v", f"-I{INCLUDE}"]
    jobs = []  # (object, command); the device units compile concurrently
    # The fused build also takes the approximate divide / square root and flushes
    # denormals; the slab scan's division stays IEEE (__fdiv_rn) in both builds.
    for unit in ("ix_kernels", "ix_pool", "ix_wavefront", "ix_metrics", "ix_display"):
        for variant, flags in (("exact", ["-DIX_EXACT=1", "-fmad=false"]),
                               ("fast", ["-DIX_EXACT=0", "-fmad=true", "-prec-div=false",
                                         "-prec-sqrt=false", "-ftz=true"])):
            obj = os.path.join(BUILD_DIR, f"{unit}_{variant}.o")
            jobs.append((obj, common + flags + ["-c", os.path.join(CSRC, unit + ".cu"), "-o", obj]))
    for unit in ("ix_probe", "ix_fixed", "ix_noalloc", "ix_radiance", "ix_surrogate", "ix_umma", "ix_image_metrics"):
        obj = os.path.join(BUILD_DIR, unit + ".o")
        jobs.append((obj, common + ["-c", os.path.join(CSRC, unit + ".cu"), "-o", obj]))
    procs = [(obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
             for obj, cmd in jobs]
    objs, logs, errors = [], [], []
    for obj, proc in procs:
        _, err = proc.communicate()
        logs.append(err)
        if proc.returncode != 0:
            errors.append(err)
        objs.append(obj)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors))
    cuda_inc = os.path.join(_cuda_home(nvcc), "include")
    for unit in ("ix_backend", "ix_dispatch", "ix_display_host", "ix_radiance_host", "ix_design"):
        host_obj = os.path.join(BUILD_DIR, unit + ".o")
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall",
               f"-I{INCLUDE}", f"-I{cuda_inc}", "-c", os.path.join(CSRC, unit + ".cpp"), "-o", host_obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed:\n" + r.stderr)
        objs.append(host_obj)
    tmp = OUT + ".tmp"
    cmd = [nvcc, "-shared", *ARCH, "-o", tmp, *objs, "-cudart", "static", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr)
    os.replace(tmp, OUT)
    with open(os.path.join(BUILD_DIR, "ptxas.log"), "w") as f:
        f.write("\n".join(logs))
    if verbose:
        print("\n".join(logs))
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
