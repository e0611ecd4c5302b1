"""Build the native parts of biobloom_b200 in-tree.

  biobloom_b200/lib/libbbt.so          CUDA kernels + C ABI (include/bbt.h)
  biobloom_b200/bin/biobloomcategorizer    CLI over the C ABI (Bloom filters)
  biobloom_b200/bin/biobloommicategorizer  CLI over the C ABI (miBF, include/bbt_mibf.h)

Device code is compiled for sm_100a only.  Objects go to biobloom_b200/_build/
and are rebuilt when a source or header is newer.
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "lib", "libbbt.so")
BIN = os.path.join(PKG, "bin")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Build settings of the kernels (for example "-DBBT_HIT_READS_ALL=1"), space
# separated; objects are rebuilt by date only, so clear _build/ after a change.
DEFINES = os.environ.get("BBT_BUILD_DEFINES", "").split()
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
          "-Xcompiler", "-fPIC,-fopenmp,-O3,-Wall", "-ccbin", "/usr/bin/g++"] + DEFINES
LIB_SOURCES = ["classify.cu", "score.cu", "dust.cu", "twopass.cu", "bucketed.cu", "api.cu", "noalloc.cu", "gather_rate.cu", "maker.cu", "mibf.cu",
               "mibf_make.cu", "formats.cpp", "pack.cpp", "fastx.cpp", "synth.cpp", "mibf_host.cpp",
               "mibf_pipeline.cpp", "server.cpp"]
CLIS = [("biobloomcategorizer", "cli_categorizer.cpp"),
        ("biobloommicategorizer", "cli_micategorizer.cpp")]


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    inc = os.path.join(ROOT, "include")
    return hs + [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode:
        sys.stderr.write(p.stdout + p.stderr)
        raise RuntimeError("native build failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and p.stderr.strip():
        sys.stderr.write(p.stderr)
    return p


def build(verbose=False, ptxas_info=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdrs = _headers()
    objs = []
    for src in LIB_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _newer(o, [s] + hdrs) or ptxas_info:
            extra = ["-Xptxas", "-v"] if (ptxas_info and src.endswith(".cu")) else []
            _run([NVCC] + ARCH + COMMON + extra + ["-c", s, "-o", o], verbose or ptxas_info)
    if _newer(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs +
             ["-Xcompiler", "-fopenmp", "-lz", "-ccbin", "/usr/bin/g++"], verbose)
    for name, src in CLIS:
        cli = os.path.join(BIN, name)
        cli_src = os.path.join(CSRC, src)
        if _newer(cli, [cli_src, LIB] + hdrs):
            _run(["/usr/bin/g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
                  cli_src, "-o", cli, "-L" + os.path.dirname(LIB), "-lbbt",
                  "-Wl,-rpath,$ORIGIN/../lib"], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
