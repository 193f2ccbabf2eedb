"""Builds libscycle_b200.so in-tree with nvcc for sm_100a."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libscycle_b200.so")
SOURCES = ["capi.cu", "sbp_solver.cu", "sbp_host.cpp", "qd.cu", "infile.cpp", "noalloc.cu", "fdiag.cu", "cycle.cu",
           "cycle_host.cpp", "powerlaw.cu", "batch.cu", "adjoint.cu", "writer.cu", "ozaki.cu", "thermal_host.cpp", "thermal.cu",
           "blockchol.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", "--expt-relaxed-constexpr"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "scycle_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=True):
    """Compiles the sources in parallel (one nvcc per file) and links."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    import tempfile
    objdir = tempfile.mkdtemp(prefix="scy_build_")
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]

    def compile_one(pair):
        src, obj = pair
        cmd = [nvcc(), *NVCC_FLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        return subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=min(len(srcs), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, zip(srcs, objs)))
    for r in results:
        if r.stderr:
            sys.stderr.write(r.stderr)
    bad = [s for s, r in zip(srcs, results) if r.returncode != 0]
    if bad:
        raise subprocess.CalledProcessError(1, "nvcc", "failed: %s" % ", ".join(bad))
    cmd = [nvcc(), *NVCC_FLAGS, "-shared", "-o", LIB + ".tmp", *objs, "-lcudart", "-lcublas", "-lcusolver"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        try:
            os.remove(o)
        except OSError:
            pass
    try:
        os.rmdir(objdir)
    except OSError:
        pass
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
