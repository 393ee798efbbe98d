"""Builds the native libraries of the package in-tree.

    python -m vectisdb_b200.build          # libvgpu.so (CUDA, sm_100a) + libvgpu_datagen.so

libvgpu.so is the engine behind include/vgpu.h: nvcc for sm_100a, CUDA runtime linked statically,
NVRTC dynamically, and no link-time dependency on libcuda (driver entry points are resolved at run
time), so the library loads on a machine without a GPU. Objects go to vectisdb_b200/_build/.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
CUDA = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA / "bin" / "nvcc")

ENGINE_SOURCES = [
    "abi.cpp",
    "plan.cpp",
    "runtime.cpp",
    "sha256.cpp",
    "codegen.cpp",
    "cost_model.cpp",
    "column_cache.cpp",
    "kernels.cu",
    "executor.cu",
    "batch.cu",
    "server.cpp",
    "stream_pipeline.cu",
    "shard.cu",
    "noalloc.cu",
    "translator.cpp",
    "ingest.cpp",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-Wall,-Wno-unused-function",
    "-I", str(ROOT / "include"), "-I", str(CSRC),
]


def _embed_device_lib() -> Path:
    src = (CSRC / "device_lib.cuh").read_text()
    delim = "VGPUEMBED"
    assert f"){delim}\"" not in src
    out = BUILD / "device_lib_embed.inc"
    text = f"static const char kDeviceLibSource[] = R\"{delim}(\n{src}\n){delim}\";\n"
    if not out.exists() or out.read_text() != text:
        out.write_text(text)
    return out


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {cmd[-1]}")


def build_engine(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    embed = _embed_device_lib()
    headers = list(CSRC.glob("*.hpp")) + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "vgpu.h", embed]
    objs, jobs = [], []
    for name in ENGINE_SOURCES:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        objs.append(obj)
        if _stale(obj, [src] + headers):
            cmd = [NVCC] + NVCC_FLAGS + ["-I", str(BUILD), f'-DVGPU_CUDA_LIB_DIR="{CUDA / "lib64"}"', "-c", str(src),
                                         "-o", str(obj)]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        list(ex.map(_run, jobs))
    lib = PKG / "libvgpu.so"
    if jobs or _stale(lib, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", str(lib)] + [str(o) for o in objs] +
             ["-ldl"])
    if verbose:
        print(f"built {lib}")
    return lib


def build_datagen(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    src = CSRC / "datagen.cpp"
    lib = PKG / "libvgpu_datagen.so"
    if _stale(lib, [src]):
        _run(["g++", "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", "-std=c++17",
              "-ffp-contract=off", "-o", str(lib), str(src)])
    if verbose:
        print(f"built {lib}")
    return lib


def main() -> None:
    build_engine(verbose=True)
    build_datagen(verbose=True)


if __name__ == "__main__":
    main()
