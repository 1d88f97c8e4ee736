"""In-tree build of libmc.so (sm_100a) and the dosefgpu_driftcorr CLI.

    python -m motioncorr1exp_b200.build            # build what is stale
    python -m motioncorr1exp_b200.build --force    # rebuild everything
    python -m motioncorr1exp_b200.build --sanitize address
        # host code instrumented by AddressSanitizer, into lib_asan/ (for
        # hunting host memory errors; load it from an instrumented program,
        # e.g. tests/native/batch_stress.cpp, with
        # ASAN_OPTIONS=protect_shadow_gap=0 so CUDA can map its memory)

Outputs go to motioncorr1exp_b200/lib/ (git-ignored, shipped with the tree).
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
LIB = os.path.join(HERE, "lib")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]

LIB_SOURCES = ["mc_kernels.cu", "mc_fwd.cu", "mc_fwd_raw.cu", "mc_fwd_dif.cu", "mc_pair.cu", "mc_sum.cu", "mc_fsc.cu", "mc_stretch.cu", "mc_plan.cu",
               "mc_solve.cu", "mc_noalloc.cu", "lsq.cpp", "mc_batch.cpp", "stack_io.cpp", "tiff_read.cpp"]
LIB_HEADERS = ["kernels.cuh", "kcommon.cuh", "fft_engine.cuh", "f2ops.cuh", "dft_gen.cuh", "codelets_gen.cuh", "lsq.h",
               "tiff_read.h"]
CLI_SOURCES = ["cli/dosefgpu_driftcorr.cpp", "cli/mrc_file.cpp"]
CLI_HEADERS = ["cli/mrc_file.h"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd[:3])} ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False, sanitize: str = "") -> str:
    lib = os.path.join(HERE, "lib_asan") if sanitize else LIB
    san = ["-Xcompiler", f"-fsanitize={sanitize}", "-Xcompiler", "-fno-omit-frame-pointer"] if sanitize else []
    os.makedirs(lib, exist_ok=True)
    objdir = os.path.join(lib, "obj")
    os.makedirs(objdir, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in LIB_HEADERS] + [os.path.join(INCLUDE, "mc.h")]
    objs, jobs = [], []
    for src in LIB_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc()] + ARCH + NVCC_FLAGS + san + ["-I", INCLUDE, "-I", CSRC, "-c", s, "-o", o]
            if ptxas_info and s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if s.endswith(".cpp"):
                cmd = [nvcc(), "-O3", "-std=c++17", "-Xcompiler", "-fPIC"] + san + ["-I", INCLUDE, "-I", CSRC,
                                                                                    "-x", "c++", "-c", s, "-o", o]
            jobs.append(cmd)
    # translation units compile in parallel (the kernel file dominates)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, c, verbose or ptxas_info) for c in jobs]:
            f.result()
    so = os.path.join(lib, "libmc.so")
    if force or _stale(so, objs):
        _run([nvcc()] + ARCH + san + ["-shared", "-o", so] + objs + ["-lcudart", "-lz", "-lpthread"], verbose)
    if sanitize:
        return so
    cli = os.path.join(LIB, "dosefgpu_driftcorr")
    cli_src = [os.path.join(CSRC, c) for c in CLI_SOURCES]
    if all(os.path.exists(c) for c in cli_src):
        deps = cli_src + [os.path.join(CSRC, h) for h in CLI_HEADERS] + [so, os.path.join(INCLUDE, "mc.h")]
        if force or _stale(cli, deps):
            cxx = os.environ.get("CXX", "g++")
            _run([cxx, "-O2", "-std=c++17", "-I", INCLUDE, "-I", os.path.join(CSRC, "cli")] + cli_src +
                 ["-L", LIB, "-lmc", "-Wl,-rpath,$ORIGIN", "-o", cli], verbose)
    return so


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers / spills per kernel")
    ap.add_argument("--sanitize", default="", help="e.g. address: instrumented host code into lib_asan/")
    a = ap.parse_args()
    print(build(a.force, a.verbose, a.ptxas_info, a.sanitize))


if __name__ == "__main__":
    main()
