"""Builds libtortoise_b200.so in-tree with nvcc for sm_100a.

Usage: python -m tortoise_b200.build   (or tortoise_b200.build.build()).
The enumeration kernel is compiled with --fmad=false so that its
floating-point filters round like the reference's unfused C++.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libtortoise_b200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
          "-I" + os.path.join(HERE, "..", "include"), "--expt-relaxed-constexpr"]
SOURCES = {
    "tb_api.cu": [],
    "tb_enumerate.cu": ["--fmad=false"],
    "tb_collision.cu": [],
    "tb_drift.cu": [],
    "tb_dp45.cu": [],
    "tb_tensor.cu": [],
    "tb_static_scratch.cu": [],
    "tb_vjp.cu": [],
    "tb_adjoint.cu": [],
    "tb_shard.cu": [],
    "tb_constraints.cu": [],
    "tb_theta.cu": [],
    "tb_probe.cu": [],
    "tb_stream.cu": [],
}


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(verbose=False, extra=(), out=OUT, build_dir=BUILD):
    """Compiles every source (in parallel, one nvcc per source) and links
    the shared library `out`."""
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(build_dir, exist_ok=True)
    cmds, objs = [], []
    for src, flags in SOURCES.items():
        obj = os.path.join(build_dir, src.replace(".cu", ".o"))
        cmds.append([nvcc(), *ARCH, *COMMON, *flags, *extra, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    # the largest sources first, so the slowest compiles start at once
    order = sorted(range(len(cmds)), key=lambda k: -os.path.getsize(cmds[k][-3]))
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for f in [pool.submit(subprocess.check_call, cmds[k]) for k in order]:
            f.result()
    cmd = [nvcc(), *ARCH, "-shared", "-o", out, *objs, "-lcudart", "-ldl"]
    if verbose:
        print(" ".join(cmd))
    subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, extra=[a for a in sys.argv[1:] if a != "-v"])
