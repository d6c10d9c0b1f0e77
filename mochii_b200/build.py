"""Build libmochii_gpu.so in-tree with nvcc for sm_100a.

    python -m mochii_b200.build        (or mochii_b200.build.build())

The device code is compiled with -fmad=false: the FP64 cell-walk geometry
and the source-energy inversion must round exactly as the FP64 source
expressions do (no fused multiply-add contraction), which is what makes
leaf sequences and sampled energies bit-identical to the CPU restatement.
The balance kernels (balance.cu) are checked against the restatement to
the solvers' tolerances, not bit for bit, and are compiled with contraction
(fewer instructions in the thermal solve).
"""
import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libmochii_gpu.so")

SOURCES = ["api.cu", "transport.cu", "balance.cu", "diffuse.cu", "band.cpp", "params.cpp", "thermal_setup.cpp", "species_setup.cpp",
           "octree_setup.cpp", "dust_setup.cpp", "dust_temp.cu", "mlp.cu", "output.cpp", "peel.cpp",
           "refine.cpp", "refine_dev.cu", "spectrum.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FMA_SOURCES = {"balance.cu"}   # tolerance-checked FP64 solves: fused multiply-add allowed


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_rebuild():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "mochii_gpu.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_rebuild():
        return LIB
    nvcc = nvcc_path()
    hostcxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    common = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "-ccbin", hostcxx, "-I", INCLUDE, "-I", CSRC] + ARCH
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        flags = [("-fmad=true" if f == "-fmad=false" and src in FMA_SOURCES else f) for f in common]
        cmd = [nvcc, "-c", os.path.join(CSRC, src), "-o", obj] + flags
        if src.endswith(".cpp"):
            cmd = [nvcc, "-x", "cu", "-c", os.path.join(CSRC, src), "-o", obj] + flags
        if verbose:
            print(" ".join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # the translation units are independent: compile them concurrently
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
            if verbose and r.stderr:
                sys.stderr.write(r.stderr)
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-shared", "-o", tmp] + objs + ARCH + ["-ccbin", hostcxx, "-lcudart", "-ldl"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
