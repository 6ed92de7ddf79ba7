"""Build the in-tree native libraries.

    python sph-cpp_b200/build.py            # product + oracle (+ reference oracle when its sources exist)

Products (all git-ignored, all travel with the repository snapshot):
  sph-cpp_b200/lib/libpbf_b200.so   the CUDA PBF step for sm_100a (C ABI of include/pbf.h)
  oracle/_build/libpbf_oracle.so    the CPU restatement used as the parity checker
  oracle/_ref/libpbf_ref*.so        the reference's own sources, compiled (only where they exist)
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
LIB = PKG / "lib" / "libpbf_b200.so"
APP = PKG / "lib" / "pbf_run"
ORACLE_LIB = ROOT / "oracle" / "_build" / "libpbf_oracle.so"
# The reference's source tree: PBF_REFERENCE_ROOT, else the read-only checkout
# this build script is run beside; absent on machines that only use the
# prebuilt oracle/_ref libraries.
REF_SOURCES = Path(os.environ.get("PBF_REFERENCE_ROOT", "/root/reference"))

NVCC_ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["csrc/pbf_cuda.cu"]
HOST_SOURCES = ["csrc/pbf_host.cpp"]
# every header the library's sources include: all of csrc/ and include/
DEPS = sorted(str(f.relative_to(PKG)) for f in (PKG / "csrc").glob("*") if f.suffix in (".cuh", ".h")) + \
    ["../include/pbf.h"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx() -> str:
    # The system gcc toolchain (with libgomp); a CXX from the environment may lack it.
    for c in ("/usr/bin/g++", shutil.which("g++") or ""):
        if c and Path(c).exists():
            return c
    raise RuntimeError("no g++ found")


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources if s.exists())


def _run(cmd: list[str], cwd: Path) -> None:
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, cwd=cwd, check=True)


def build_product(force: bool = False, verbose_ptxas: bool = False) -> Path:
    srcs = [PKG / s for s in CUDA_SOURCES + HOST_SOURCES + DEPS]
    if not force and not _stale(LIB, srcs):
        return LIB
    LIB.parent.mkdir(parents=True, exist_ok=True)
    obj_dir = PKG / "_build"
    obj_dir.mkdir(exist_ok=True)
    host_obj = obj_dir / "pbf_host.o"
    _run([_host_cxx(), "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-c", str(PKG / HOST_SOURCES[0]),
          "-o", str(host_obj)], PKG)
    cmd = [_nvcc(), *NVCC_ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-ccbin", _host_cxx(), "-o", str(LIB), *[str(PKG / s) for s in CUDA_SOURCES], str(host_obj)]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    _run(cmd, PKG)
    return LIB


def build_app(force: bool = False) -> Path:
    """The headless driver (apps/pbf_run.cpp), linked against libpbf_b200.so."""
    src = PKG / "apps" / "pbf_run.cpp"
    deps = [src, ROOT / "include" / "pbf.h", ROOT / "include" / "pbf_particles.hpp", LIB]
    if force or _stale(APP, deps):
        _run([_host_cxx(), "-O2", "-std=c++17", str(src), "-I", str(ROOT / "include"), "-L", str(LIB.parent),
              "-lpbf_b200", "-Wl,-rpath,$ORIGIN", "-o", str(APP)], PKG)
    return APP


def build_oracle(force: bool = False) -> Path:
    src = ROOT / "oracle" / "pbf_oracle.c"
    if force or _stale(ORACLE_LIB, [src, ROOT / "include" / "pbf.h"]):
        ORACLE_LIB.parent.mkdir(parents=True, exist_ok=True)
        gcc = "/usr/bin/gcc" if Path("/usr/bin/gcc").exists() else "gcc"
        _run([gcc, "-O2", "-std=c11", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o",
              str(ORACLE_LIB), "-lm"], ROOT)
    return ORACLE_LIB


def build_reference(force: bool = False) -> bool:
    """Compile the reference's own sources where they exist (this container);
    on machines without them the prebuilt libraries under oracle/_ref are used."""
    if not (REF_SOURCES / "Simulation" / "Source" / "particles.h").exists():
        return (ROOT / "oracle" / "_ref" / "libpbf_ref.so").exists()
    args = ["make", "-C", str(ROOT / "oracle" / "ref_build"), f"REF={REF_SOURCES}"]
    if force:
        args.insert(1, "-B")
    _run(args, ROOT)
    return True


def main(argv: list[str]) -> int:
    force = "--force" in argv
    build_product(force=force, verbose_ptxas="--ptxas" in argv)
    build_app(force=force)
    build_oracle(force=force)
    build_reference(force=force)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
