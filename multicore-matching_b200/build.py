"""Build recipe for the in-tree native libraries.

    libmmatch.so  CUDA kernels + C ABI (include/mm_match.h), sm_100a only
    libmtc.so     reference-compatible C++ classes (include/mtc/*.h) over the C ABI
    libmmgen.so   deterministic synthetic graph generators (host, OpenMP)

Everything is compiled in place (the .so files travel with the source tree)
and rebuilt only when a source or header is newer than its output.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
OBJ = PKG / "_build"

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
CXX = shutil.which("g++") or "g++"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC,-fvisibility=hidden", f"-I{INCLUDE}", f"-I{CSRC}"]
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-fvisibility=hidden", f"-I{INCLUDE}",
             "-I/usr/local/cuda/include"]

CUDA_SOURCES = ["mm_capi.cu", "mm_pull.cu", "mm_push.cu", "mm_noalloc.cu", "mm_check.cu", "mm_contract.cu"]
MTC_SOURCES = ["mtc_graph.cpp", "mtc_matching.cpp", "mtc_gpu.cpp"]


def _newer(out: Path, deps: list[Path]) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def _headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.rglob("*.h"))


def build_mmatch(verbose: bool = False) -> Path:
    out = PKG / "libmmatch.so"
    OBJ.mkdir(exist_ok=True)
    objs = []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = OBJ / (src + ".o")
        if _newer(o, [s] + _headers() + [Path(__file__)]):
            _run([NVCC, *NVCC_FLAGS, "-c", s, "-o", o], verbose)
        objs.append(o)
    script = OBJ / "mmatch.map"
    script.write_text("{ global: mm_*; local: *; };\n")
    if _newer(out, objs):
        # static cudart, and a version script: only the mm_* C ABI is exported
        # (template instantiations from C++ headers would otherwise leak as weak symbols)
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", out, *objs,
              "-Xlinker", "--exclude-libs,ALL", "-Xlinker", f"--version-script={script}"], verbose)
    return out


def build_mtc(verbose: bool = False) -> Path:
    out = PKG / "libmtc.so"
    srcs = [CSRC / s for s in MTC_SOURCES if (CSRC / s).exists()]
    if not srcs:
        return out
    libmm = PKG / "libmmatch.so"
    if _newer(out, srcs + _headers() + [libmm]):
        # C++14: Graph::random_shuffle draws its permutation with std::random_shuffle
        # (removed in C++17), exactly as the reference does
        flags = [f for f in CXX_FLAGS if not f.startswith("-std=")] + ["-std=c++14"]
        _run([CXX, *flags, "-fvisibility=default", "-shared", "-o", out, *srcs,
              f"-L{PKG}", "-lmmatch", f"-Wl,-rpath,$ORIGIN",
              "-L/usr/local/cuda/lib64", "-lcudart"], verbose)
    return out


def build_mmgen(verbose: bool = False) -> Path:
    out = PKG / "libmmgen.so"
    src = CSRC / "graphgen.cpp"
    if _newer(out, [src]):
        _run([CXX, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-fvisibility=hidden",
              "-o", out, src], verbose)
    return out


def build_oracle(verbose: bool = False, ref_src: str | None = None) -> None:
    """The CPU checker: the restatement always; the reference's own matchers too
    when ref_src (or the environment's MM_REFERENCE_SRC) names the reference's
    src/ directory."""
    ref_src = ref_src or os.environ.get("MM_REFERENCE_SRC")
    target = ["ref"] if ref_src and (Path(ref_src) / "matchtbb.cu").exists() else ["all"]
    env = dict(os.environ)
    env.pop("CC", None)
    env.pop("CXX", None)
    cmd = ["make", "-s", "-C", str(ROOT / "oracle"), *target] + ([f"REF_SRC={ref_src}"] if target == ["ref"] else [])
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, env=env)


def build_all(verbose: bool = False, ref_src: str | None = None) -> None:
    build_mmatch(verbose)
    build_mtc(verbose)
    build_mmgen(verbose)
    build_oracle(verbose, ref_src)


if __name__ == "__main__":
    build_all(verbose="-v" in sys.argv)
