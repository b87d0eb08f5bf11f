"""Build recipe for the oracle (checker) libraries.

  oracle/liborc.so               abf_oracle.c (gcc): k-way merge, mixed-format
                                 restatement, CPU baseline
  oracle/libwgen.so              the seeded workload generator
                                 (adabool_b200/csrc/abf_gen.cpp + gen_shim.cpp,
                                 g++), so that the reference's timing leg
                                 generates the benchmark data without loading
                                 the product library
  oracle/_ref/libref_build.so    the reference's own ivf_list::BuildFrom,
                                 compiled with g++ from the reference sources
                                 (host memory only, no GPU needed)
  oracle/_ref/libref_harness.so  the reference's single-query driver with its
                                 CPU ground truth and GPU kernels, compiled with
                                 nvcc for sm_100a from the reference sources

The two _ref libraries are built only where the reference source tree is
present: REFERENCE_ROOT if set, else a checkout named `reference` beside
this repository's directory. It is read in place and nothing is copied from
it. The reference headers miss <array>/<memory> includes, which are added
with -include.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REF_OUT = HERE / "_ref"
LIBORC = HERE / "liborc.so"
LIBWGEN = HERE / "libwgen.so"
REF_BUILD = REF_OUT / "libref_build.so"
REF_HARNESS = REF_OUT / "libref_harness.so"
REFERENCE_ROOT = Path(os.environ.get("REFERENCE_ROOT") or HERE.parent.parent / "reference")
SHIM = ["-include", "array", "-include", "memory"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle build failed: " + " ".join(map(str, cmd)))


def _stale(out: Path, srcs) -> bool:
    return not out.exists() or any(Path(s).stat().st_mtime > out.stat().st_mtime for s in srcs)


def build_orc() -> Path:
    srcs = [HERE / "abf_oracle.c", HERE / "abf_oracle.h"]
    if _stale(LIBORC, srcs):
        _run(["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-Wall", "-D_POSIX_C_SOURCE=200809L",
              str(HERE / "abf_oracle.c"), "-o", str(LIBORC), "-lpthread"])
    return LIBORC


def build_wgen() -> Path:
    csrc = HERE.parent / "adabool_b200" / "csrc"
    srcs = [csrc / "abf_gen.cpp", HERE / "gen_shim.cpp", csrc / "abf_internal.h",
            HERE.parent / "include" / "abf_workload.h", HERE.parent / "include" / "adabool.h"]
    if _stale(LIBWGEN, srcs):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-Wall", "-march=x86-64-v2", str(csrc / "abf_gen.cpp"),
              str(HERE / "gen_shim.cpp"), "-o", str(LIBWGEN), "-lpthread"])
    return LIBWGEN


def reference_present() -> bool:
    return (REFERENCE_ROOT / "src" / "AdaBool" / "inverted_list.h").exists()


def build_ref(with_gpu: bool = True) -> list[Path]:
    """Builds the reference-derived libraries; returns those that exist."""
    if reference_present():
        REF_OUT.mkdir(exist_ok=True)
        cuda_inc = "/usr/local/cuda/include"
        ref_src = REFERENCE_ROOT / "src" / "AdaBool"
        if _stale(REF_BUILD, [HERE / "ref_build.cpp"]):
            _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", f"-I{ref_src}", f"-I{cuda_inc}",
                  "-include", "cuda_runtime.h", *SHIM, str(HERE / "ref_build.cpp"), "-o", str(REF_BUILD)])
        if with_gpu and _stale(REF_HARNESS, [HERE / "ref_harness.cu"]):
            nvcc = "/usr/local/cuda/bin/nvcc" if Path("/usr/local/cuda/bin/nvcc").exists() else "nvcc"
            _run([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC",
                  "-shared", f"-I{REFERENCE_ROOT / 'test'}", f"-I{ref_src}", *SHIM, str(HERE / "ref_harness.cu"),
                  "-o", str(REF_HARNESS), "-lstdc++fs"])
    return [p for p in (REF_BUILD, REF_HARNESS) if p.exists()]


def build_all(with_gpu: bool = True):
    build_orc()
    build_wgen()
    return build_ref(with_gpu)


if __name__ == "__main__":
    print(build_orc(), build_wgen(), build_ref(with_gpu="--no-gpu" not in sys.argv))
