"""Build the vpfft_b200 native library in-tree.

    python -m vpfft_b200.build [--force] [--ptxas-verbose]

Compiles vpfft_b200/csrc/*.cu and *.cpp with nvcc for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) into vpfft_b200/lib/libvpfft_b200.so.
The CUDA runtime is linked statically, so the library needs only the NVIDIA
driver at run time.  Objects are rebuilt when a source or header is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "lib", "obj")
LIB = os.path.join(PKG, "lib", "libvpfft_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-I", INCLUDE,
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the vpfft_b200 CUDA library cannot be built")


def _deps() -> float:
    hdrs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hdrs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return max((os.path.getmtime(h) for h in hdrs), default=0.0)


# The line-transform units are built without floating-point contraction: their
# product-sums are written out with fused multiply-adds (fmad), so every
# compiled copy of a pass -- single-grid tiles and each batched tile family --
# performs the same operations and gives the same bits.
NO_CONTRACT = {"fft.cu", "fft_fixed_small.cu", "fft_fixed_large.cu", "fft_tma.cu"}


def _compile(src: str, force: bool, verbose_ptxas: bool) -> tuple[str, str]:
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), _deps())):
        return obj, ""
    extra = ["--fmad=false"] if os.path.basename(src) in NO_CONTRACT else []
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force: bool = False, verbose_ptxas: bool = False, quiet: bool = True) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    logs = []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        futs = [ex.submit(_compile, s, force, verbose_ptxas) for s in srcs]
        objs = []
        for f in futs:
            o, log = f.result()
            objs.append(o)
            if log:
                logs.append(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas and logs:
        with open(os.path.join(PKG, "lib", "ptxas.log"), "w") as fh:
            fh.write("\n".join(logs))
    if not quiet:
        print(LIB)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    build(force=a.force, verbose_ptxas=a.ptxas_verbose, quiet=False)
    return 0


if __name__ == "__main__":
    sys.exit(main())
