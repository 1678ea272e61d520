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

ENGINE_SRC = ["engine.cpp", "plan.cpp", "kernels.cu"]
DRIVER_SRC = ["driver.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    deps = list(sources) + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    deps.append(os.path.join(HERE, "..", "include", "libgint.h"))
    return any(os.path.getmtime(s) > t for s in deps if os.path.exists(s))


def build_engine(force=False, verbose=False):
    out = os.path.join(LIB, "libgint_b200.so")
    srcs = [os.path.join(CSRC, f) for f in ENGINE_SRC]
    if force or _stale(out, srcs):
        os.makedirs(LIB, exist_ok=True)
        cmd = [NVCC] + ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                               "-Xptxas", "-v", "-o", out] + srcs + ["-lcudart"]
        log = _run(cmd)
        if verbose:
            print(log)
    return out


def build_driver(force=False):
    out = os.path.join(LIB, "libgint_driver.so")
    srcs = [os.path.join(CSRC, f) for f in DRIVER_SRC]
    if force or _stale(out, srcs):
        os.makedirs(LIB, exist_ok=True)
        _run([HOSTCXX, "-O2", "-std=c++17", "-fPIC", "-shared", "-o", out] + srcs + ["-ldl"])
    return out


def build_all(force=False):
    return build_engine(force), build_driver(force)


if __name__ == "__main__":
    print(build_engine(force=True, verbose=True))
    print(build_driver(force=True))
