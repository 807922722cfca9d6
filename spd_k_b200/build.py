"""Build libspdk_cuda.so in-tree with nvcc for sm_100a.

The parity (FP64) kernels are compiled with -fmad=false and the host code
with -ffp-contract=off: no product is fused into a sum anywhere, so the
arithmetic rounds exactly like the reference's x86-64 CPU build. The FP32
precision form's translation units (FP32_SOURCES) are compiled with FMA
contraction and FP32 division/square root to within 2 ulp (its FP64
islands are unaffected): that form makes no bitwise claim.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libspdk_cuda.so")
SOURCES = ["spdk_hydro.cu", "spdk_select_2d_low.cu", "spdk_select_2d_high.cu", "spdk_select_3d.cu",
           "spdk_select_f32_2d.cu", "spdk_select_f32_3d.cu",
           "spdk_noalloc.cu", "spdk_proto.cu", "spdk_induction.cu", "spdk_induction2d.cu", "spdk_tc_study.cu", "spdk_mlp.cu", "spdk_batch_f64.cu",
           "spdk_batch_f32.cu", "spdk_batch_host.cu", "spdk_checkpoint.cu", "spdk_conserved.cu", "spdk_setup.cpp",
           "spdk_host_api.cpp"]
FP32_SOURCES = {"spdk_select_f32_2d.cu", "spdk_select_f32_3d.cu", "spdk_batch_f32.cu", "spdk_tc_study.cu"}
HEADERS = ["spdk_physics.cuh", "spdk_kernels.cuh", "spdk_fallback.cuh", "spdk_kernelset.cuh", "spdk_setup.h",
           "spdk_reflayout.cuh", "spdk_learned_impl.h", "spdk_batch.cuh", "spdk_hydro_impl.h", "spdk_viscous.cuh", "spdk_picard2d.cuh"]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def flags(extra=(), fmad=False):
    return [
        "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
        *(["-fmad=true", "-prec-div=false", "-prec-sqrt=false"] if fmad else ["-fmad=false"]),
        "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
        "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
        "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills",
        *extra,
    ]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "driver", "spdk_run.cpp"))
    deps += [os.path.join(ROOT, "include", h) for h in ("spdk.h", "spdk_proto.h", "spdk_induction.h", "spdk_learned.h", "spdk_batch.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False, jobs=None):
    if not force and not stale():
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs, procs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [nvcc, *flags(fmad=src in FP32_SOURCES), "-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    for p, src in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{out.decode()[-6000:]}")
        if verbose and out:
            print(out.decode()[-3000:])
    tmp = LIB + ".tmp"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    os.replace(tmp, LIB)
    # the athinput-driven driver executable, linked against the library
    drv = os.path.join(HERE, "spdk_run")
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"),
           os.path.join(HERE, "driver", "spdk_run.cpp"), "-o", drv + ".tmp",
           "-L" + HERE, "-l:libspdk_cuda.so", "-Wl,-rpath,$ORIGIN"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("driver build failed:\n" + r.stdout + r.stderr)
    os.replace(drv + ".tmp", drv)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
