"""Build libqsim.so (sm_100a) in-tree with nvcc.

    python -m quict_b200.build            # compile if sources are newer
    python -m quict_b200.build --force    # always recompile
    python -m quict_b200.build --ptxas-v  # print ptxas register/smem usage
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
OBJDIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libqsim.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "--split-compile", "0"]  # device code optimised in parallel (the fused kernels are large)


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


# the persistent batch kernel as relocatable device code (linked at run time
# with generated register-stage functions), embedded in the library
RDC_SRC = os.path.join(CSRC, "rdc", "batch_dev.cu")
RDC_CUBIN = os.path.join(OBJDIR, "batch_dev.cubin")
RDC_C = os.path.join(OBJDIR, "batch_dev_cubin.c")
RDC_OBJ = os.path.join(OBJDIR, "batch_dev_cubin.o")


def embed_cubin(cubin: str, csrc: str, obj: str) -> None:
    """Write the cubin as a C byte array (qs_batch_dev_cubin) and compile it."""
    data = open(cubin, "rb").read()
    with open(csrc, "w") as f:
        f.write("/* generated by quict_b200/build.py from csrc/rdc/batch_dev.cu */\n")
        f.write(f"const unsigned long long qs_batch_dev_cubin_size = {len(data)}ull;\n")
        f.write("__attribute__((aligned(16))) const unsigned char qs_batch_dev_cubin[] = {\n")
        for i in range(0, len(data), 32):
            f.write(",".join(str(b) for b in data[i:i + 32]) + ",\n")
        f.write("};\n")
    r = subprocess.run(["gcc", "-O0", "-fPIC", "-c", csrc, "-o", obj], capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("compile of the embedded batch cubin failed")


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = sources()
    hdrs = headers()
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(OBJDIR, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or ptxas_verbose or _stale(o, [s] + hdrs):
            cmd = [nvcc(), *ARCH, *FLAGS, "-I", INCLUDE, "-c", s, "-o", o]
            if ptxas_verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    rdc_stale = force or ptxas_verbose or _stale(RDC_CUBIN, [RDC_SRC] + hdrs)
    if rdc_stale:
        cmd = [nvcc(), "-arch=sm_100a", "-rdc=true", "-cubin", "-O3", "-lineinfo", "-std=c++17",
               "--expt-relaxed-constexpr", "-I", INCLUDE, RDC_SRC, "-o", RDC_CUBIN]
        if ptxas_verbose:
            cmd += ["-Xptxas", "-v"]
        jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for cmd, r in ex.map(run, jobs):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError(f"nvcc failed: {' '.join(cmd)}")
            if ptxas_verbose or (r.stderr.strip() and not quiet):
                sys.stderr.write(r.stderr)
    if rdc_stale or _stale(RDC_OBJ, [RDC_CUBIN]):
        embed_cubin(RDC_CUBIN, RDC_C, RDC_OBJ)
    objs.append(RDC_OBJ)
    if force or jobs or _stale(LIB, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("link of libqsim.so failed")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, ptxas_verbose=a.ptxas_v))


if __name__ == "__main__":
    main()
