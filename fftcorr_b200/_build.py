"""Builds the fftcorr_b200 CUDA library in-tree for sm_100a.

    python -m fftcorr_b200._build [--reference DIR]

Outputs fftcorr_b200/libfftcorr_b200.so (git-ignored; it travels with the
source tree).  When the reference source tree is available (--reference, or
$FFTCORR_REFERENCE) its D12 wavelet table is generated into csrc/_gen/ first
(see csrc/gen_d12.cc); without it the library is built without the D12
scheme and reports FC_ERR_UNSUPPORTED for it.

A rebuild is decided by content: a SHA-256 over every source and header,
the generated table, the compiler flags and the nvcc version is stored
beside the library (libfftcorr_b200.so.sha256) and compared on each build,
so a library built from other sources is never reused.
"""
import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "_gen")
LIB = os.path.join(HERE, "libfftcorr_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
DEFAULT_REFERENCE = os.environ.get("FFTCORR_REFERENCE")

SOURCES = ["fc_core.cu", "fc_hist.cu", "fc_assign.cu", "fc_fused.cu", "fc_corr.cu",
           "fc_batch.cu", "fc_catalog.cu", "fc_serve.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++20",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "--expt-relaxed-constexpr",
]
# Products are rounded one by one like the reference's FP64 code, except in
# the FFT passes, where fused multiply-adds only change rounding inside the
# transform (which differs from FFTW's anyway) and halve the arithmetic.
NO_FMAD = ["-fmad=false"]
FMAD_OK = {"fc_fused.cu"}


def _run(cmd, cwd=None):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=cwd)


def generate_d12(reference):
    """Writes csrc/_gen/d12_table.inc from the reference's d12.h, if present."""
    out = os.path.join(GEN, "d12_table.inc")
    header = os.path.join(reference, "cc", "particle_mesh", "d12.h") if reference else None
    if header is None or not os.path.exists(header):
        return os.path.exists(out)
    os.makedirs(GEN, exist_ok=True)
    exe = os.path.join(GEN, "gen_d12")
    _run(["g++", "-std=c++11", "-O0", "-I", os.path.join(reference, "cc"),
          os.path.join(CSRC, "gen_d12.cc"), "-o", exe])
    table = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    if os.path.exists(out):
        with open(out) as f:
            if f.read() == table:
                return True
    tmp = out + ".tmp"
    with open(tmp, "w") as f:
        f.write(table)
    os.replace(tmp, out)
    return True


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


STAMP = LIB + ".sha256"


def _nvcc_version():
    try:
        return subprocess.run([NVCC, "--version"], check=True, capture_output=True,
                              text=True).stdout
    except (OSError, subprocess.CalledProcessError):
        return "nvcc unavailable"


def content_hash():
    """SHA-256 of everything the library is built from."""
    h = hashlib.sha256()
    deps = sources() + sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC)
                              if f.endswith((".cuh", ".h")))
    deps.append(os.path.join(HERE, "..", "include", "fc_api.h"))
    gen = os.path.join(GEN, "d12_table.inc")
    if os.path.exists(gen):
        deps.append(gen)
    for d in deps:
        h.update(os.path.basename(d).encode() + b"\0")
        with open(d, "rb") as f:
            h.update(f.read())
    h.update(repr((NVCC_FLAGS, NO_FMAD, sorted(FMAD_OK), SOURCES)).encode())
    h.update(_nvcc_version().encode())
    return h.hexdigest()


def needs_rebuild():
    if not os.path.exists(LIB) or not os.path.exists(STAMP):
        return True
    with open(STAMP) as f:
        return f.read().strip() != content_hash()


def build(reference=DEFAULT_REFERENCE, force=False, verbose_ptxas=False):
    generate_d12(reference)
    if not force and not needs_rebuild():
        if cli_needs_rebuild():
            build_cli()
        return LIB
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    extra = ["-Xptxas", "-v"] if verbose_ptxas else []

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        fmad = [] if os.path.basename(src) in FMAD_OK else NO_FMAD
        _run([NVCC, *NVCC_FLAGS, *fmad, *extra, "-I", CSRC, "-c",
              src, "-o", obj])
        return obj

    with ThreadPoolExecutor(max(1, min(len(SOURCES), os.cpu_count() or 1))) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB + ".tmp"
    _run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
          *objs, "-o", tmp, "-L", os.path.join(CUDA_HOME, "lib64"), "-lcufft",
          "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")])
    os.replace(tmp, LIB)
    with open(STAMP, "w") as f:
        f.write(content_hash() + "\n")
    build_cli()
    return LIB


CLI = os.path.join(HERE, "bin", "fftcorr")
CLI_STAMP = CLI + ".sha256"


def _cli_hash():
    h = hashlib.sha256()
    for d in (os.path.join(CSRC, "fftcorr_cli.cc"),
              os.path.join(HERE, "..", "include", "fc_api.h")):
        with open(d, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def cli_needs_rebuild():
    if not os.path.exists(CLI) or not os.path.exists(CLI_STAMP):
        return True
    with open(CLI_STAMP) as f:
        return f.read().strip() != _cli_hash()


def build_cli():
    """The `fftcorr` command-line driver (csrc/fftcorr_cli.cc) on the library."""
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    _run(["g++", "-O2", "-std=c++17", os.path.join(CSRC, "fftcorr_cli.cc"),
          "-o", CLI, "-L", HERE, "-lfftcorr_b200", "-Wl,-rpath,$ORIGIN/.."])
    with open(CLI_STAMP, "w") as f:
        f.write(_cli_hash() + "\n")
    return CLI


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.reference, a.force, a.ptxas_v))


if __name__ == "__main__":
    main()
