"""Build recipe of librevsim.so (the C-ABI CUDA library) for sm_100a, in-tree.

Each .cu file under csrc/ is compiled separately with nvcc (in parallel) and
linked into rev-sim_b200/librevsim.so.  No JIT cache is involved, so the built
library travels with the source tree.
"""

import hashlib
import os
import subprocess
import tempfile
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
# Object files go to a scratch directory outside the source tree (only the linked
# library lives in-tree).
BUILD = os.path.join(tempfile.gettempdir(), "revsim_build_" + hashlib.sha1(HERE.encode()).hexdigest()[:10])
LIB = os.path.join(HERE, "librevsim.so")
SOURCES = ["rs_api.cu", "rs_step.cu", "rs_nlist.cu", "rs_loss.cu", "rs_probe.cu", "sw_kernels.cu",
           "sw_api.cu"] + [
    f"rs_step_{p}_{f}.cu" for p in "fd" for f in ("lj", "dexp", "buck", "ljsc", "buff", "ljmlp")] + [
    f"rs_half_{f}.cu" for f in ("lj", "dexp", "buck", "ljsc", "buff", "ljmlp")] + [
    "rs_mlp.cu", "rs_mlp_tc.cu", "rs_energy.cu", "rs_barostat.cu", "gas_kernels.cu", "gas_api.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
         "--expt-relaxed-constexpr"]


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    files += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(f) for f in files)


def _compile(src, extra):
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(force=False, verbose=False, extra=()):
    """Compile csrc/*.cu for sm_100a and link librevsim.so; returns its path."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, list(extra)), SOURCES))
    if verbose:
        for _, err in results:
            if err:
                print(err, file=sys.stderr)
    objs = [o for o, _ in results]
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    extra = ["-Xptxas", "-v"] if "-v" in sys.argv else []
    print(build(force=True, verbose=bool(extra), extra=extra))
