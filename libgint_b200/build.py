"""Builds the native libraries in-tree (libgint_b200/lib), for sm_100a.

  libgint_b200.so    the engine: C-ABI (include/libgint.h), host batcher, CUDA kernels
  libgint_driver.so  workload generator / C0 fitter / C-ABI replayer (the stand-in caller)
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC = os.environ.get("NVCC", "nvcc")
HOSTCXX = "g++"

# (source, extra flags, object name); prim3.cu and group3.cu are compiled once per part so the
# generated classes compile in parallel
PRIM3_PARTS = 8
GROUP3_PARTS = 4
# engine.cpp holds the team-collective calls (orphaned OpenMP constructs bound to the caller's team)
ENGINE_OBJS = [("engine.cpp", ["-Xcompiler", "-fopenmp"], "engine.o"), ("plan.cpp", [], "plan.o"), ("kernels.cu", [], "kernels.o")] + \
    [("prim3.cu", [f"-DPRIM3_PART={i}"], f"prim3_{i}.o") for i in range(PRIM3_PARTS)] + \
    [("group3.cu", [f"-DGROUP3_PART={i}"], f"group3_{i}.o") for i in range(GROUP3_PARTS)]
DRIVER_SRC = ["driver.cpp"]
OBJDIR = os.path.join(HERE, "_build")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "libgint.h"))
    return hs


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = list(sources) + _headers()
    return any(os.path.getmtime(s) > t for s in deps if os.path.exists(s))


def build_engine(force=False, verbose=False):
    """nvcc each translation unit to an object (in parallel), then link the shared library."""
    from concurrent.futures import ThreadPoolExecutor
    out = os.path.join(LIB, "libgint_b200.so")
    os.makedirs(OBJDIR, exist_ok=True)
    jobs = []
    for src, flags, obj in ENGINE_OBJS:
        s, o = os.path.join(CSRC, src), os.path.join(OBJDIR, obj)
        if force or _stale(o, [s]):
            jobs.append([NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                                         "-Xptxas", "-v"] + flags + ["-c", s, "-o", o])
    logs = []
    if jobs:
        with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
            logs = list(ex.map(_run, jobs))
    objs = [os.path.join(OBJDIR, o) for _, _, o in ENGINE_OBJS]
    if force or jobs or _stale(out, objs):
        os.makedirs(LIB, exist_ok=True)
        logs.append(_run([NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-lcudart", "-lgomp"]))
    if verbose:
        print("\n".join(logs))
    return out


def build_driver(force=False):
    out = os.path.join(LIB, "libgint_driver.so")
    srcs = [os.path.join(CSRC, f) for f in DRIVER_SRC]
    if force or _stale(out, srcs):
        os.makedirs(LIB, exist_ok=True)
        _run([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-o", out] + srcs + ["-ldl"])
    return out


def build_all(force=False):
    return build_engine(force), build_driver(force)


if __name__ == "__main__":
    print(build_engine(force=True, verbose=True))
    print(build_driver(force=True))
