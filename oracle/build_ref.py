"""Build recipe for oracle/_ref (test infrastructure, not part of the product).

Compiles the reference's own CPU fitness path -- its Simulator, op, state,
model and evaluator sources, unchanged, from the reference checkout -- plus
oracle/ref_harness.cpp into two shared libraries:

  oracle/_ref/libgrn_ref.so     -O2 -ffp-contract=off: the parity build, whose
                                FP64 results the tests compare bit for bit
                                with the restatement (oracle/grn_oracle.cpp)
  oracle/_ref/libgrn_ref_o3.so  -O3 -march=x86-64-v3: the timed build, used by
                                bench.py's CPU baseline and reference arm

Qt and Eigen are not installed; oracle/shims/qt provides the part of their
API those files use.  The classes around the path that live in the
reference's database layer (Search, SimParams, Experiment, MorphologyImage)
come from oracle/shims/ref.  Those stand-in headers take precedence over the
reference's own headers of the same names through g++'s -I- (quote includes
are then searched in the directories given before -I-, and not in the
including file's own directory).

The reference checkout is read from $GRN_REFERENCE_ROOT (default
/root/reference).  Without it nothing is built and the functions return None;
the built libraries travel with the repository to machines that lack it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT_DIR, "libgrn_ref.so")
LIB_O3 = os.path.join(OUT_DIR, "libgrn_ref_o3.so")

REF_SOURCES = [
    "Src/Simulator/modelsimulator.cpp",
    "Src/Simulator/simop.cpp",
    "Src/Simulator/simopand.cpp",
    "Src/Simulator/simopor.cpp",
    "Src/Simulator/simophillact.cpp",
    "Src/Simulator/simophillrep.cpp",
    "Src/Simulator/simopzero.cpp",
    "Src/Simulator/simopone.cpp",
    "Src/Simulator/simopcopy.cpp",
    "Src/Simulator/simstate.cpp",
    "Src/Simulator/simulator.cpp",
    "Src/Model/model.cpp",
    "Src/Model/modelprod.cpp",
    "Src/Model/modellink.cpp",
    "Src/Search/evaluatormorphogens.cpp",
]

PARITY_FLAGS = ["-O2", "-fno-fast-math", "-ffp-contract=off"]
TIMED_FLAGS = ["-O3", "-march=x86-64-v3"]


def reference_root():
    return os.environ.get("GRN_REFERENCE_ROOT", "/root/reference")


def _own_files():
    files = [os.path.join(HERE, "ref_harness.cpp"), os.path.abspath(__file__),
             os.path.join(ROOT, "include", "grn_gpu.h")]
    for sub in ("shims/qt", "shims/ref"):
        for d, _, names in os.walk(os.path.join(HERE, sub)):
            files += [os.path.join(d, n) for n in names]
    return files


def _stdlib_quote_dirs():
    """Directories of the C++ library's own quote includes.  libstdc++'s
    parallel-algorithm headers include each other with quotes relative to
    their directory, which -I- stops searching; naming that directory again
    after -I- restores it."""
    out = subprocess.run(["g++", "-xc++", "-E", "-v", "-"], input="", capture_output=True,
                         text=True).stderr
    dirs = []
    for line in out.splitlines():
        d = os.path.join(line.strip(), "pstl")
        if line.startswith(" ") and os.path.isfile(os.path.join(d, "execution_defs.h")):
            dirs += ["-I", d]
    return dirs


def _command(src_root, flags, out):
    src = os.path.join(src_root, "Src")
    inc = ["-I", os.path.join(HERE, "shims", "ref"), "-I-"] + _stdlib_quote_dirs() + [
           "-I", os.path.join(HERE, "shims", "qt"),
           "-I", src, "-I", os.path.join(src, "Simulator"),
           "-I", os.path.join(src, "Model"), "-I", os.path.join(src, "Search"),
           "-I", os.path.join(ROOT, "include")]
    sources = [os.path.join(src_root, s) for s in REF_SOURCES] + [
        os.path.join(HERE, "ref_harness.cpp")]
    return (["g++", "-std=c++17", "-fPIC", "-shared", "-pthread", "-w"] + flags + inc +
            ["-o", out] + sources)


def build(force=False, verbose=False):
    """Builds both libraries if the reference checkout is present; returns the
    parity library's path, or None when the checkout is absent and no library
    was built before."""
    src_root = reference_root()
    if not os.path.isdir(os.path.join(src_root, "Src", "Simulator")):
        return LIB if os.path.exists(LIB) else None
    os.makedirs(OUT_DIR, exist_ok=True)
    deps = _own_files() + [os.path.join(src_root, s) for s in REF_SOURCES]
    for flags, out in ((PARITY_FLAGS, LIB), (TIMED_FLAGS, LIB_O3)):
        if not force and os.path.exists(out):
            t = os.path.getmtime(out)
            if all(os.path.getmtime(d) <= t for d in deps):
                continue
        cmd = _command(src_root, flags, out)
        if verbose:
            print(" ".join(cmd))
        # g++ notes that -I- is obsolete once per source; show its output only
        # when the build fails.
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("building %s failed" % out)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
