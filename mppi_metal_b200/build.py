"""Builds libmppi_b200.so in-tree (mppi_metal_b200/lib/).

    python -m mppi_metal_b200.build        # or build() from Python

Steps
  1. embed the device sources (csrc/device/*.cuh, mppi_launch.h) as string
     literals for the runtime NVRTC compile (csrc/embedded_sources.inc);
  2. nvcc -gencode arch=compute_100a,code=sm_100a the ahead-of-time kernels;
  3. g++ the host runtime (backend, NVRTC module cache, driver, C facades);
  4. link one shared library against the static CUDA runtime and NVRTC.
Targets sm_100a only.  Rebuilds only what changed (mtime based).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
DEVICE = CSRC / "device"
OBJ = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libmppi_b200.so"
INCLUDE = ROOT / "include"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

EMBED = ["mppi_prelude.cuh", "mppi_launch.h", "mppi_gelu.cuh", "mppi_kernels.cuh"]
HOST_SOURCES = ["backend.cpp", "nvrtc_module.cpp", "driver.cpp", "driver_c.cpp"]
CUDA_SOURCES = ["static_kernels.cu", "noalloc.cu", "proposal_mlp.cu"]
DELIM = "mppi_b200_src"


def _newer(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _embed() -> Path:
    out = CSRC / "embedded_sources.inc"
    deps = [DEVICE / n for n in EMBED]
    if not _newer(out, deps + [Path(__file__)]):
        return out
    parts = ["// Generated by mppi_metal_b200/build.py from csrc/device/ -- do not edit.\n",
             "static const EmbeddedFile kEmbeddedFiles[] = {\n"]
    for name in EMBED:
        text = (DEVICE / name).read_text()
        if f"){DELIM}\"" in text:
            raise RuntimeError(f"{name} contains the raw-string delimiter")
        parts.append(f'  {{"{name}", R"{DELIM}({text}){DELIM}"}},\n')
    parts.append("};\n")
    out.write_text("".join(parts))
    return out


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    """Compile (incrementally) and return the path of libmppi_b200.so."""
    if not Path(NVCC).exists():
        raise RuntimeError(f"nvcc not found at {NVCC}")
    OBJ.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    _embed()
    headers = list(DEVICE.glob("*")) + list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.inc")) \
        + list(INCLUDE.rglob("*.h*"))
    common = ["-O3", "-std=c++17", f"-I{INCLUDE}", f"-I{CSRC}"]
    jobs = []
    objs = []
    for src in CUDA_SOURCES:
        o = OBJ / (src + ".o")
        objs.append(o)
        if _newer(o, [CSRC / src] + headers):
            cmd = [NVCC, *ARCH, "-lineinfo", *common, "-Xcompiler", "-fPIC", "-c",
                   str(CSRC / src), "-o", str(o)]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    for src in HOST_SOURCES:
        o = OBJ / (src + ".o")
        objs.append(o)
        if _newer(o, [CSRC / src] + headers):
            jobs.append(["g++", *common, "-fPIC", "-Wall", "-Wno-unused-function",
                         f"-I{CUDA_HOME / 'include'}", "-c", str(CSRC / src), "-o", str(o)])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for cmd in jobs:
                if verbose:
                    print(" ".join(cmd), file=sys.stderr)
            list(ex.map(_run, jobs))
    if jobs or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs),
              f"-L{CUDA_HOME / 'lib64'}", "-lnvrtc",
              "-Xlinker", f"-rpath,{CUDA_HOME / 'lib64'}"])
        shutil.move(str(tmp), str(LIB))
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv))
