"""Build the sm_100a CUDA library in-tree: scrs_b200/_lib/libscrs_b200.so.

    python -m scrs_b200.build

nvcc compiles every translation unit for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with the CUDA runtime linked
statically, so the library shares the driver's primary context with any
other runtime (torch) in the process.
"""
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT = HERE / "_lib" / "libscrs_b200.so"
SOURCES = ["mxk_kernels.cu", "afft.cu", "engines.cu", "batch.cu", "noalloc.cu", "server.cu", "tune.cu", "jit.cu"]
GEN = HERE / "_lib" / "gen"
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr", "-I", str(GEN)]
# headers the run-time compiler (jit.cu) is given: name as #included -> file
JIT_HEADERS = [("mxk_spec.cuh", CSRC / "mxk_spec.cuh"), ("mxk_device.cuh", CSRC / "mxk_device.cuh"),
               ("common.cuh", CSRC / "common.cuh"), ("kernels.cuh", CSRC / "kernels.cuh")]
# NVRTC has no C library headers; the device code needs only these types
JIT_SHIMS = [("stdint.h", "#pragma once\n"
              "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long long int64_t;\n"
              "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
              "typedef unsigned long long uint64_t; typedef unsigned long uintptr_t;\n")]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def generate():
    """Regenerate the PTX jump tables when their generator is newer."""
    gen, out = CSRC / "gen_brx.py", CSRC / "brx_dispatch.cuh"
    if not out.exists() or out.stat().st_mtime < gen.stat().st_mtime:
        subprocess.run([sys.executable, str(gen)], check=True)


def generate_jit_sources():
    """_lib/gen/jit_sources.inc: the device headers as C++ raw strings, which
    jit.cu hands to NVRTC with every specialised kernel."""
    GEN.mkdir(parents=True, exist_ok=True)
    out = GEN / "jit_sources.inc"
    items = [(n, p.read_text()) for n, p in JIT_HEADERS] + JIT_SHIMS
    lines = ["// generated by scrs_b200/build.py from the device headers; do not edit", "namespace {"]
    lines.append("const char* const kJitHeaderNames[] = {" + ", ".join(f'"{n}"' for n, _ in items) + "};")
    lines.append("const char* const kJitHeaderTexts[] = {")
    for _, text in items:
        assert ")SCRS_SRC\"" not in text
        lines.append('R"SCRS_SRC(' + text + ')SCRS_SRC",')
    lines.append("};")
    lines.append(f"constexpr int kJitHeaderCount = {len(items)};")
    lines.append("}  // namespace")
    body = "\n".join(lines) + "\n"
    if not out.exists() or out.read_text() != body:
        out.write_text(body)


def build(verbose: bool = False, force: bool = False) -> Path:
    generate()
    generate_jit_sources()
    srcs = [CSRC / s for s in SOURCES if (CSRC / s).exists()]
    deps = srcs + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [HERE.parent / "include" / "scrs_gpu.h"]
    if OUT.exists() and not force and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    obj_dir = HERE / "_lib" / "obj"
    obj_dir.mkdir(parents=True, exist_ok=True)
    objs = []
    procs = []
    for s in srcs:
        o = obj_dir / (s.stem + ".o")
        objs.append(o)
        cmd = [nvcc(), *FLAGS, "-c", str(s), "-o", str(o)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    failed = False
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out)
        if p.returncode != 0:
            failed = True
    if failed:
        raise RuntimeError("nvcc compilation failed")
    link = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-cudart", "static",
            *[str(o) for o in objs], "-ldl", "-o", str(OUT)]
    subprocess.run(link, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
