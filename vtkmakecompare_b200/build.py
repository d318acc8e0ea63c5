"""Build libnsegpu.so (the CUDA kernels + C-ABI) in-tree for sm_100a.

Every kernel file except the FFT file is compiled with --fmad=false so the
stencil, line-solver and level-set arithmetic rounds operation by operation
like the reference's Fortran build; the FFT file keeps FMA contraction.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libnsegpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-Xcompiler", "-Wall"]
SOURCES = {
    "runtime.cu": ["--fmad=false"],
    "k_stencil.cu": ["--fmad=false"],
    "k_line.cu": ["--fmad=false"],
    "k_levelset.cu": ["--fmad=false"],
    "k_lines_exact.cu": ["--fmad=false"],
    "k_lines_fast.cu": [],
    "k_lines_part.cu": [],
    "k_rhs_fast.cu": [],
    "k_rhs_f32.cu": ["--fmad=false"],
    "k_fft.cu": [],
    "k_poisson2d.cu": [],
    "noalloc.cu": [],
    "tma.cu": [],
    "fortran_io.cu": [],
    "k_adjoint.cu": ["--fmad=false"],
    "adjoint.cu": [],
}


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _needs(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, "common.cuh"), os.path.join(CSRC, "k_lines.cuh"),
               os.path.join(CSRC, "fft_core.cuh"), os.path.join(CSRC, "tma.cuh"),
               os.path.join(CSRC, "k_rhs_fast.cuh"),
               os.path.join(CSRC, "k_adjoint.cuh"),
               os.path.join(HERE, "..", "include", "nsegpu.h")]
    jobs = []
    objs = []
    for src, flags in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if _needs(o, [s] + headers + [__file__]):
            cmd = [nvcc()] + ARCH + COMMON + list(flags) + list(extra) + ["-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for out in ex.map(run, jobs):
            if verbose and out.strip():
                print(out)
    if jobs or not os.path.exists(LIB) or _needs(LIB, objs):
        run([nvcc()] + ARCH + ["-shared", "-o", LIB] + objs)
    return LIB


if __name__ == "__main__":
    extra = sys.argv[1:]
    print(build(verbose=True, extra=extra))
