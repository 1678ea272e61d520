"""Runs one K build of the reference CUDA library in a child process.

The reference library calls exit() on a CUDA API error (for example its batch memset is
rejected for some batch sizes), which would end the whole test session; running it in a child
process turns that into one failed test. Usage:
    python tests/ref_runner.py OUT.npy MAX_MEM_MB WORKLOAD_JSON
WORKLOAD_JSON holds {"name": ..., **overrides} as passed to libgint_b200.workload.Workload.
"""
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def reference_K(spec, max_mem_mb, timeout=600):
    """K (packed) of the reference CUDA build for Workload(**spec), and its wall time in ms."""
    import tempfile
    import numpy as np
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "K.npy")
        r = subprocess.run([sys.executable, os.path.abspath(__file__), out, str(max_mem_mb), json.dumps(spec)],
                           capture_output=True, text=True, timeout=timeout, cwd=ROOT)
        if r.returncode != 0 or not os.path.exists(out):
            raise RuntimeError(f"reference build failed (rc={r.returncode}): {(r.stdout + r.stderr)[-400:]}")
        K = np.load(out)
        ms = float(np.load(out + ".ms.npy"))
    return K, ms


def main(argv):
    import numpy as np
    sys.path.insert(0, ROOT)
    sys.path.insert(0, HERE)
    from conftest import REF_GINT_SO
    from libgint_b200.workload import Api, Session, Workload
    out, max_mem, spec = argv[1], int(argv[2]), json.loads(argv[3])
    name = spec.pop("name")
    wl = Workload(name, **spec)
    s = Session(Api(REF_GINT_SO), wl, max_mem_mb=max_mem)
    K, ms, _ = s.build_K()
    s.close()
    np.save(out + ".ms.npy", np.array(ms))
    np.save(out, K)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
