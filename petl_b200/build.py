"""Builds petl_b200/libpetl.so from petl_b200/csrc (nvcc, sm_100a).

    python -m petl_b200.build        # or petl_b200.build.build()

The library is built in-tree so that it travels with the repository to a GPU
machine.  Every translation unit is compiled separately and in parallel;
host code is compiled without floating-point contraction so that the host
restatements of the reference's float expressions round exactly as the
reference's host code does.
"""
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libpetl.so")
OBJ = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx():
    # a plain system g++ (some images export a CXX without OpenMP support)
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return "g++"


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _compile(src, verbose=False, extra=()):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(HERE, "..", "include", f) for f in os.listdir(os.path.join(HERE, "..", "include"))]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj, ""
    cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler",
           "-fPIC,-fopenmp,-ffp-contract=off", "--expt-relaxed-constexpr", "-c", src, "-o", obj, *extra]
    if src.endswith(".cpp"):
        cmd[cmd.index("-c")] = "-x"
        cmd.insert(cmd.index("-x") + 1, "cu")
        cmd.insert(cmd.index("cu") + 1, "-c")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj, (r.stdout + r.stderr) if verbose else ""


def build(verbose=False, jobs=None, extra=()):
    """Compile every csrc translation unit for sm_100a and link libpetl.so."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose, extra), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            if log:
                print(log)
    newest = max(os.path.getmtime(o) for o in objs)
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < newest:
        cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs,
               "-Xcompiler", "-fopenmp", "-lgomp"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    v = "-v" in sys.argv
    extra = ["-Xptxas", "-v"] if "--ptxas" in sys.argv else []
    print(build(verbose=v or bool(extra), extra=extra))
