"""Builds lible_b200/liblible_b200.so (sm_100a) in-tree with nvcc.

Objects go to lible_b200/_build/; each translation unit is rebuilt when it or any header it
includes (transitively, #include "...") is newer than its object.  Instantiation files are
regenerated first.

    python -m lible_b200.build [-j N]
"""
import argparse
import concurrent.futures as cf
import glob
import os
import re
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "liblible_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# the embedded sm_100a images are compressed (-compress-all): about 3x smaller objects and library
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++20", "--expt-relaxed-constexpr", "-Xfatbin", "-compress-all",
                     "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-O3", "-I" + CSRC]


def nvcc():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def sources():
    sys.path.insert(0, CSRC)
    import gen_instances  # noqa: E402
    gen_instances.main()
    srcs = [os.path.join(CSRC, f) for f in ("host_math.cpp", "host_basis.cpp", "engine.cu", "peak.cu", "noalloc.cu",
                                            "ri_k.cu", "oneel.cu", "eri_special.cu", "capi.cpp")]
    srcs += sorted(glob.glob(os.path.join(CSRC, "gen", "*.cu")))
    return srcs


_INCLUDE = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def local_deps(path, seen=None):
    """The source file and every header it includes with #include "..." (transitively)."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as fh:
        for inc in _INCLUDE.findall(fh.read()):
            local_deps(os.path.join(os.path.dirname(path), inc), seen)
    return seen


def newest_dep(src):
    return max(os.path.getmtime(d) for d in local_deps(src))


def obj_path(src):
    rel = os.path.relpath(src, CSRC).replace(os.sep, "_")
    return os.path.join(OUT_DIR, rel + ".o")


def compile_one(src, verbose=False):
    obj = obj_path(src)
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep(src):
        return obj, None
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [nvcc(), "-x", "cu"] + NVCC_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr + r.stdout
    if verbose:
        print("compiled", os.path.relpath(src, HERE), flush=True)
    return obj, None


def build(jobs=None, verbose=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    # objects built with other flags are stale
    stamp = os.path.join(OUT_DIR, "flags.txt")
    flags = " ".join(NVCC_FLAGS)
    if not os.path.exists(stamp) or open(stamp).read() != flags:
        for o in glob.glob(os.path.join(OUT_DIR, "*.o")):
            os.remove(o)
        with open(stamp, "w") as fh:
            fh.write(flags)
    srcs = sources()
    jobs = jobs or os.cpu_count() or 4
    objs, errors = [], []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        for obj, err in ex.map(lambda s: compile_one(s, verbose), srcs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errors)[:20000])
    for o in glob.glob(os.path.join(OUT_DIR, "*.o")):
        if o not in objs:
            os.remove(o)  # object of a source that no longer exists
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcusolver", "-lcublas"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr + r.stdout)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    args = ap.parse_args()
    print(build(args.j, verbose=True))
