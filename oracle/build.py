"""Build recipes for the oracle (test infrastructure; nothing in the product loads these).

1. oracle/liblux_oracle.so: the plain-C restatement in oracle/lux_oracle.c.
2. oracle/liblux_pt64.so: the FP64 path-tracing oracle in oracle/pt64.c.
3. oracle/_ref/libluxref.so: the reference's own host code.
4. oracle/_ref/libluxrefgpu.so: the reference's own GPU LBVH (bvh/gpu_bvh.cu,
   bvh/bvh_overlap.cu) behind oracle/ref_gpu_harness.cu, compiled with nvcc for sm_100a.
7. oracle/_ref/libluxref_dmath.so: item 3 with oracle/rounded_double_math.h
   force-included (the rounding-isolation test's reference side).
6. oracle/_ref/libluxshim.so: the drop-in shims (lux_b200/integration/) compiled
   against the reference's headers and called through its own types
   (oracle/ref_shim_harness.cpp), linked to lux_b200/liblux_gpu.so.
5. oracle/_ref/libluxrefpt.so: the reference's own GPU wavefront path tracer
   (integrator/wavefront_*.cu, scene/prepared_scene.cu, bvh/gpu_bvh.cu,
   light/light_distribution.cpp) behind oracle/ref_pt_gpu_harness.cu, compiled with nvcc
   for sm_100a, one object per translation unit.

Compiles, in place and without the reference's build system, the handful of
reference translation units the CPU path needs (integrator/cpu_path_tracer.cpp,
light/light_distribution.cpp, scene/prepared_scene_cpu.cpp, and util/obj_loader.cpp for
the asset scenes; everything else on the path is header-only) together with oracle/ref_harness.cpp.  Output goes only to
oracle/_ref/.  Test infrastructure: nothing in the product loads this library.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("LUX_REFERENCE_ROOT", "/root/reference")
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libluxref.so")
ORACLE_OUT = os.path.join(HERE, "liblux_oracle.so")
PT64_OUT = os.path.join(HERE, "liblux_pt64.so")

REF_SOURCES = [
    "src/integrator/cpu_path_tracer.cpp",
    "src/light/light_distribution.cpp",
    "src/scene/prepared_scene_cpu.cpp",
    "src/util/obj_loader.cpp",
]

# The reference's Release configuration: -O3, x86-64 baseline ISA (SSE2, so no FMA
# contraction is possible), IEEE semantics (no -ffast-math).
CXXFLAGS = ["-std=c++20", "-O3", "-fPIC", "-ffp-contract=off", "-pthread"]


def _stale(out, inputs):
    if not os.path.exists(out):
        return True
    return os.path.getmtime(out) < max(os.path.getmtime(p) for p in inputs)


def build_oracle(force=False):
    """Compile the C restatement (single precision, no contraction)."""
    srcs = [os.path.join(HERE, "lux_oracle.c")]
    if force or _stale(ORACLE_OUT, srcs):
        cmd = ["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
               "-o", ORACLE_OUT, *srcs, "-lm"]
        subprocess.run(cmd, check=True)
    return ORACLE_OUT


def build_pt64(force=False):
    """Compile the FP64 path-tracing oracle (double precision, pthreads)."""
    srcs = [os.path.join(HERE, "pt64.c")]
    if force or _stale(PT64_OUT, srcs):
        cmd = ["gcc", "-std=c11", "-O3", "-fPIC", "-shared", "-pthread", "-ffp-contract=off",
               "-o", PT64_OUT, *srcs, "-lm"]
        subprocess.run(cmd, check=True)
    return PT64_OUT


def build_ref(force=False):
    """Compile the reference harness; returns None when the reference is absent."""
    src_dir = os.path.join(REF_ROOT, "src")
    if not os.path.isdir(src_dir):
        return None
    harness = os.path.join(HERE, "ref_harness.cpp")
    inputs = [harness] + [os.path.join(REF_ROOT, s) for s in REF_SOURCES]
    deps = inputs + [os.path.join(HERE, "ref_scene_desc.h"),
                     os.path.join(HERE, "..", "include", "lux_gpu.h")]
    if not force and not _stale(OUT, deps):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", *CXXFLAGS, "-shared", "-I", src_dir, "-I", HERE, "-o", OUT, *inputs]
    subprocess.run(cmd, check=True)
    return OUT


REF_DMATH_OUT = os.path.join(OUT_DIR, "libluxref_dmath.so")


def build_ref_dmath(force=False):
    """The reference harness again with oracle/rounded_double_math.h force-included: the
    reference's float sinf/cosf/powf/acosf/atan2f evaluated in double and rounded, as
    lux_b200/liblux_gpu_dmath.so evaluates them (the rounding-isolation test's pair)."""
    src_dir = os.path.join(REF_ROOT, "src")
    if not os.path.isdir(src_dir):
        return None
    harness = os.path.join(HERE, "ref_harness.cpp")
    header = os.path.join(HERE, "rounded_double_math.h")
    inputs = [harness] + [os.path.join(REF_ROOT, s) for s in REF_SOURCES]
    deps = inputs + [header, os.path.join(HERE, "ref_scene_desc.h"),
                     os.path.join(HERE, "..", "include", "lux_gpu.h")]
    if not force and not _stale(REF_DMATH_OUT, deps):
        return REF_DMATH_OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", *CXXFLAGS, "-shared", "-include", header, "-I", src_dir, "-I", HERE,
           "-o", REF_DMATH_OUT, *inputs]
    subprocess.run(cmd, check=True)
    return REF_DMATH_OUT


REF_GPU_OUT = os.path.join(OUT_DIR, "libluxrefgpu.so")
REF_GPU_SOURCES = ["src/bvh/bvh_overlap.cu"]
REF_GPU_HEADERS = ["src/bvh/gpu_bvh.cu", "src/bvh/gpu_bvh.cuh", "src/bvh/bvh_device.cuh"]
# The reference's stock CUDA configuration (CMakeLists.txt: C++20, Release -O3,
# LUX_ENABLE_CUDA=1); nvcc's default contraction is kept, as the reference builds.
NVCCFLAGS = ["-std=c++20", "-O3", "-DLUX_ENABLE_CUDA=1",
             "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC"]


def build_ref_gpu(force=False):
    """Compile the reference's GPU LBVH harness; None when the reference is absent."""
    src_dir = os.path.join(REF_ROOT, "src")
    if not os.path.isdir(src_dir):
        return None
    harness = os.path.join(HERE, "ref_gpu_harness.cu")
    inputs = [harness] + [os.path.join(REF_ROOT, s) for s in REF_GPU_SOURCES]
    deps = inputs + [os.path.join(REF_ROOT, s) for s in REF_GPU_HEADERS]
    if not force and not _stale(REF_GPU_OUT, deps):
        return REF_GPU_OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["nvcc", *NVCCFLAGS, "-shared", "-I", src_dir, "-o", REF_GPU_OUT, *inputs]
    subprocess.run(cmd, check=True)
    return REF_GPU_OUT


REF_PT_OUT = os.path.join(OUT_DIR, "libluxrefpt.so")
REF_PT_SOURCES = [
    "src/integrator/wavefront_kernels.cu",
    "src/integrator/wavefront_pt.cu",
    "src/integrator/wavefront_runtime.cu",
    "src/integrator/wavefront_scheduler.cu",
    "src/scene/prepared_scene.cu",
    "src/bvh/gpu_bvh.cu",
    "src/light/light_distribution.cpp",
]


def _ref_headers(src_dir):
    out = []
    for root, _, files in os.walk(src_dir):
        out += [os.path.join(root, f) for f in files if f.endswith((".h", ".cuh"))]
    return out


def build_ref_pt_gpu(force=False):
    """Compile the reference's GPU wavefront tracer harness; None when the reference is
    absent.  Each translation unit becomes one object (in parallel), linked into one
    library whose only exported symbols are the harness's refpt_* entry points."""
    import concurrent.futures

    src_dir = os.path.join(REF_ROOT, "src")
    if not os.path.isdir(src_dir):
        return None
    harness = os.path.join(HERE, "ref_pt_gpu_harness.cu")
    sources = [harness] + [os.path.join(REF_ROOT, s) for s in REF_PT_SOURCES]
    deps = sources + [os.path.join(HERE, "ref_scene_desc.h"),
                      os.path.join(HERE, "..", "include", "lux_gpu.h")] + _ref_headers(src_dir)
    if not force and not _stale(REF_PT_OUT, deps):
        return REF_PT_OUT
    obj_dir = os.path.join(OUT_DIR, "refpt_obj")
    os.makedirs(obj_dir, exist_ok=True)

    def compile_one(src):
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        flags = [] if src == harness else ["-Xcompiler", "-fvisibility=hidden"]
        lang = ["-x", "cu"] if src.endswith(".cu") else []
        cmd = ["nvcc", *NVCCFLAGS, *flags, "-I", src_dir, "-I", HERE, *lang, "-c", src,
               "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"compile failed for {src}:\n{res.stderr[-4000:]}")
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(sources)) as pool:
        objs = list(pool.map(compile_one, sources))
    cmd = ["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xlinker", "--no-undefined", "-o", REF_PT_OUT, *objs]
    subprocess.run(cmd, check=True)
    return REF_PT_OUT


REF_SHIM_OUT = os.path.join(OUT_DIR, "libluxshim.so")
SHIM_DIR = os.path.join(HERE, "..", "lux_b200", "integration")
LUX_LIB_DIR = os.path.join(HERE, "..", "lux_b200")
# Reference sources the shimmed integrator factory links against (CPU scene preparation:
# the shim's integrator does not need PreparedScene::prepare_gpu).
REF_SHIM_SOURCES = [
    ("src/integrator/integrator_factory.cpp", ["-DLUX_ENABLE_CUDA=1"]),
    ("src/integrator/cpu_path_tracer.cpp", []),
    ("src/light/light_distribution.cpp", []),
    ("src/scene/prepared_scene_cpu.cpp", []),
]


def build_ref_shim(force=False):
    """Compile the drop-in shims (lux_b200/integration/) against the reference's headers,
    with oracle/ref_shim_harness.cpp and the reference sources above, linked to
    lux_b200/liblux_gpu.so; None when the reference is absent."""
    import concurrent.futures

    src_dir = os.path.join(REF_ROOT, "src")
    if not os.path.isdir(src_dir):
        return None
    include = os.path.join(HERE, "..", "include")
    shim_cpp = os.path.join(SHIM_DIR, "gpu_bvh_lux.cpp")
    shim_cu = os.path.join(SHIM_DIR, "wavefront_pt_lux.cu")
    harness = os.path.join(HERE, "ref_shim_harness.cpp")
    units = [(shim_cpp, []), (shim_cu, []), (harness, [])] + [
        (os.path.join(REF_ROOT, s), f) for s, f in REF_SHIM_SOURCES]
    deps = [u for u, _ in units] + [os.path.join(SHIM_DIR, "lux_shim.h"),
                                    os.path.join(HERE, "ref_scene_desc.h"),
                                    os.path.join(include, "lux_gpu.h")] + _ref_headers(src_dir)
    if not force and not _stale(REF_SHIM_OUT, deps):
        return REF_SHIM_OUT
    obj_dir = os.path.join(OUT_DIR, "shim_obj")
    os.makedirs(obj_dir, exist_ok=True)
    incs = ["-I", src_dir, "-I", include, "-I", SHIM_DIR, "-I", HERE]

    def compile_one(unit):
        src, flags = unit
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        if src.endswith(".cu") or src == harness:
            cmd = ["nvcc", *NVCCFLAGS, *incs, *flags, "-x", "cu", "-c", src, "-o", obj]
        else:
            cmd = ["g++", *CXXFLAGS, *incs, *flags, "-c", src, "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"compile failed for {src}:\n{res.stderr[-4000:]}")
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(units)) as pool:
        objs = list(pool.map(compile_one, units))
    cmd = ["nvcc", "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", REF_SHIM_OUT,
           *objs, "-L", LUX_LIB_DIR, "-llux_gpu", "-Xlinker", "-rpath=$ORIGIN/../../lux_b200",
           "-Xlinker", "--no-undefined"]
    subprocess.run(cmd, check=True)
    return REF_SHIM_OUT


def build(force=False):
    build_pt64(force)
    build_ref_gpu(force)
    build_ref_pt_gpu(force)
    build_ref_shim(force)
    build_ref_dmath(force)
    return build_oracle(force), build_ref(force)


if __name__ == "__main__":
    oracle_path, ref_path = build(force="--force" in sys.argv)
    print(oracle_path)
    print(ref_path if ref_path else "reference sources not present; reference harness not built")
