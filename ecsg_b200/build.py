"""Build recipe for libecsg_b200.so (sm_100a) -- in-tree, no JIT cache.

    python -m ecsg_b200.build            # library only
    python -m ecsg_b200.build --all      # + the test-side checkers under oracle/

Every kernel is compiled for sm_100a only.  interface.cu and diag.cu are built
without FMA contraction (double-precision interface solves and reductions
round like the reference); stencil.cu controls rounding with explicit
intrinsics, so its own flags do not matter for parity.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
BUILD_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "libecsg_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = {
    "stencil.cu": [],
    "stencil_v4.cu": [],
    "stencil_r.cu": ["-fmad=false"],
    "stress21.cu": ["-fmad=false"],
    "stress21_tma.cu": ["-fmad=false"],
    "vel_tma.cu": [],
    "medium.cu": [],
    "adjoint.cu": ["-fmad=false"],
    "interface.cu": ["-fmad=false"],
    "diag.cu": ["-fmad=false"],
    "api.cu": [],
    "noalloc.cu": [],
}


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _newer(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build_lib(verbose=False, force=False):
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    headers.append(os.path.join(ROOT, "include", "ecsg_b200.h"))
    objs = []
    procs = []
    for src, extra in SOURCES.items():
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        objs.append(o)
        if not force and _newer(o, [s] + headers):
            continue
        cmd = [nvcc()] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                                 "-Xptxas", "-v" if verbose else "-O3", "-c", s, "-o", o] + extra
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose:
            sys.stdout.write(out.decode())
    if force or procs or not _newer(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        subprocess.check_call(cmd)
    return LIB


CLI_DIR = os.path.join(HERE, "cli")
CLI = os.path.join(OUT_DIR, "ecsg_main")


def build_cli():
    """ecsg_main: the reference's command-line driver on the library (host C++,
    linked to libecsg_b200.so next to it)."""
    srcs = [os.path.join(CLI_DIR, f) for f in ("ecsg_main.cpp", "rsf_io.cpp")]
    deps = srcs + [os.path.join(CLI_DIR, "rsf_io.hpp"), os.path.join(ROOT, "include", "ecsg_b200.h"), LIB]
    if _newer(CLI, deps):
        return CLI
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), "-o", CLI] + srcs + \
          ["-L", OUT_DIR, "-lecsg_b200", "-Wl,-rpath,$ORIGIN", "-lpthread"]
    subprocess.check_call(cmd)
    return CLI


def build_oracle():
    """Test-side checkers: the C restatement always; the reference build
    (oracle/_ref) only where the reference sources are found (reference_dir),
    including the reference driver linked through ecsg_b200/shim (build_lib
    first)."""
    mk = os.path.join(ROOT, "oracle")
    subprocess.check_call(["make", "-s", "-C", mk, "oracle"])
    ref = reference_dir()
    if ref:
        subprocess.check_call(["make", "-s", "-C", mk, "ref", "REF=" + ref])
        # the reference driver linked against the shim and the library (needs LIB)
        subprocess.check_call(["make", "-s", "-C", mk, "shim", "REF=" + ref])


def reference_dir():
    """The reference checkout: $ECSG_REFERENCE, else a checkout named
    "reference" beside this repository; None when neither exists."""
    for d in (os.environ.get("ECSG_REFERENCE"), os.path.join(os.path.dirname(ROOT), "reference")):
        if d and os.path.isfile(os.path.join(d, "main.cpp")):
            return os.path.abspath(d)
    return None


if __name__ == "__main__":
    build_lib(verbose="-v" in sys.argv, force="--force" in sys.argv)
    build_cli()
    if "--all" in sys.argv:
        build_oracle()
    print(LIB)
