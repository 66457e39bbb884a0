"""Build recipe for lux_b200/liblux_gpu.so (sm_100a only).

Each .cu under lux_b200/csrc is compiled by nvcc for sm_100a into an object, then all
objects are linked into one shared library placed in the package directory, so the
library travels with the source tree.  `python -m lux_b200.build [--force] [-v]`.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblux_gpu.so")
CLI = os.path.join(HERE, "lux-render")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-I", os.path.join(HERE, "..", "include"),
]


# Translation units whose device arithmetic must not be contracted into FMAs (the path
# tracer restates the reference's host arithmetic operation by operation).
PER_FILE_FLAGS = {
    "wavefront.cu": ["-fmad=false"],
    "scene.cu": ["-fmad=false"],
    "server.cu": ["-fmad=false"],
}


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    out = []
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        out += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".cuh", ".h"))]
    return out


def _compile(src, verbose, obj_dir=OBJ_DIR, extra=()):
    obj = os.path.join(obj_dir, os.path.splitext(os.path.basename(src))[0] + ".o")
    if src.endswith(".cpp"):  # host-only code (the OBJ loader)
        cmd = ["g++", "-std=c++17", "-O2", "-fPIC", "-Wall",
               "-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj]
    else:
        cmd = [NVCC, *NVCC_FLAGS, *PER_FILE_FLAGS.get(os.path.basename(src), []), *extra,
               "-c", src, "-o", obj]
    if verbose and not src.endswith(".cpp"):
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed for {src}:\n{res.stderr}")
    return obj, res.stderr


def build(force=False, verbose=False):
    os.makedirs(OBJ_DIR, exist_ok=True)
    sources = _sources()
    deps = sources + _headers() + [os.path.abspath(__file__)]
    if not force and os.path.exists(LIB):
        if os.path.getmtime(LIB) >= max(os.path.getmtime(p) for p in deps):
            build_cli()
            return LIB
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose), sources))
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    objs = [o for o, _ in results]
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB, *objs,
           "-lcudart"]
    subprocess.run(cmd, check=True)
    build_cli(force=True)
    return LIB


DMATH_LIB = os.path.join(HERE, "liblux_gpu_dmath.so")
DMATH_OBJ_DIR = os.path.join(HERE, "_build_dmath")


def build_dmath(force=False):
    """The validation build liblux_gpu_dmath.so: the same sources with
    LUX_ROUNDED_DOUBLE_MATH (lux_math.cuh), whose float sinf/cosf/powf/acosf/atan2f are
    evaluated in double and rounded.  Only the rounding-isolation test loads it; it binds
    its own symbols (-Bsymbolic) so that it can sit beside liblux_gpu.so in one process."""
    os.makedirs(DMATH_OBJ_DIR, exist_ok=True)
    sources = [s for s in _sources() if s.endswith(".cu")]
    deps = sources + _headers() + [os.path.abspath(__file__)]
    if not force and os.path.exists(DMATH_LIB):
        if os.path.getmtime(DMATH_LIB) >= max(os.path.getmtime(p) for p in deps):
            return DMATH_LIB
    extra = ("-DLUX_ROUNDED_DOUBLE_MATH",)
    with concurrent.futures.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:
        results = list(pool.map(lambda s: _compile(s, False, DMATH_OBJ_DIR, extra), sources))
    objs = [o for o, _ in results]
    # The OBJ loader has no floating-point functions: the product object serves both.
    objs.append(os.path.join(OBJ_DIR, "obj.o"))
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", DMATH_LIB,
           *objs, "-lcudart", "-Xlinker", "-Bsymbolic"]
    subprocess.run(cmd, check=True)
    return DMATH_LIB


def build_cli(force=False):
    """The lux-render command line (C++20 over the C ABI), next to the library."""
    src = os.path.join(HERE, "cli", "lux_render.cpp")
    if not force and os.path.exists(CLI) and os.path.getmtime(CLI) >= max(
            os.path.getmtime(src), os.path.getmtime(LIB)):
        return CLI
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-I", os.path.join(HERE, "..", "include"), src,
           "-L", HERE, "-llux_gpu", "-Wl,-rpath,$ORIGIN", "-o", CLI]
    subprocess.run(cmd, check=True)
    return CLI


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
