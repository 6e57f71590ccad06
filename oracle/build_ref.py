"""Build recipe for oracle/_ref: the reference's own CUDA kernel sources compiled for the host.

Test infrastructure only (never imported by the product).  It reads the reference
kernels where they lie (``$SAILFISH_REFERENCE``, default: a ``reference`` checkout beside the
repository):

    modules/mod_cppkernels.cpp        -> oracle/_ref/libsfref_2d.so
    nonlinear/rhs_kernels.cpp         -> oracle/_ref/libsfref_rhs.so
    nonlinear/step3D_uv.kernels.cpp   -> oracle/_ref/libsfref_step3d.so
    modules/mod_BC.c                  -> oracle/_ref/libsfref_bc.so

Before compiling it applies the same source preprocessing the reference applies before
handing the code to NVRTC (modules/mod_operators.py:130-136: Greek identifiers are
renamed eta->E, xi->X, Delta->D, sigma->sig, then NFKD-normalised to ASCII).  The
generated sources go to oracle/_ref/src/ (git-ignored); nothing is copied into the
tracked tree.  Each library also carries the launch wrappers in oracle/ref_launch_*.cpp
(``sfref_<kernel>(nthreads, omp, args...)``), which execute the kernel once per CUDA
thread index, in order (omp <= 1) or over OpenMP threads (CPU-baseline timing only).

The reference's stencil header (modules/mod_cppkernels.h) binds reference data members to
by-value constructor parameters (e.g. ``L &expr;`` at :352 initialised from ``Expr(L _expr)``
at :360), so every interpolation/difference node reads a dead stack object: undefined
behaviour that AddressSanitizer reports as stack-use-after-return and that crashes a host
build at every optimisation level.  The generated copy of the header therefore declares
those members by value (``L expr;``), which is the value each reference aliases at the
moment it is bound; no expression, operand or evaluation order is changed.

Floating-point contraction is disabled (-ffp-contract=off) so that the results are the
IEEE-754 evaluation of each expression as written, which is what the oracle restates.

``build_native()`` compiles the same generated sources again at ``-O3 -march=native`` (with
contraction left to the compiler) into ``libsfref_<module>_native.so``, for the timed CPU
path of the reference on the machine that runs it; it needs only oracle/_ref/src, not the
reference checkout, so it can run where the benchmark runs.
"""
import os
import re
import subprocess
import sys
import unicodedata

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
MODULES = {
    "2d": ("modules/mod_cppkernels.cpp", "ref_launch_2d.cpp"),
    "rhs": ("nonlinear/rhs_kernels.cpp", "ref_launch_rhs.cpp"),
    "step3d": ("nonlinear/step3D_uv.kernels.cpp", "ref_launch_step3d.cpp"),
    "bc": ("modules/mod_BC.c", "ref_launch_bc.cpp"),
}


def reference_root():
    return os.environ.get("SAILFISH_REFERENCE",
                          os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference"))


def preprocess(code):
    # Same renaming as the reference's loader (modules/mod_operators.py:132-136).
    for a, b in (("η", "E"), ("ξ", "X"), ("Δ", "D"), ("σ", "sig")):
        code = code.replace(a, b)
    return unicodedata.normalize("NFKD", code).encode("ascii", "ignore").decode("ascii")


def patch_header(code):
    # Dangling reference members -> by-value members (see the module docstring).
    return re.sub(r"^(\s*)(L|R|OType) &(\w+);", r"\1\2 \3;", code, flags=re.M)


def lib_path(name, suffix=""):
    return os.path.join(OUT, "libsfref_%s%s.so" % (name, suffix))


def build(verbose=False, opt="-O2"):
    ref = reference_root()
    if not os.path.isdir(ref):
        if verbose:
            print("reference not present at %s; oracle/_ref not rebuilt" % ref)
        return False
    os.makedirs(os.path.join(OUT, "src"), exist_ok=True)
    hdr_src = os.path.join(ref, "modules", "mod_cppkernels.h")
    with open(hdr_src, encoding="utf-8-sig") as f:
        hdr = patch_header(preprocess(f.read()))
    hdr_gen = os.path.join(OUT, "src", "mod_cppkernels.h")
    old = open(hdr_gen).read() if os.path.exists(hdr_gen) else None
    if old != hdr:
        with open(hdr_gen, "w") as f:
            f.write(hdr)
    for name, (src_rel, launcher) in MODULES.items():
        src = os.path.join(ref, src_rel)
        with open(src, encoding="utf-8-sig") as f:
            code = preprocess(f.read())
        gen = os.path.join(OUT, "src", "%s.cpp" % name)
        with open(gen, "w") as f:
            f.write(code)
        target = lib_path(name)
        if (os.path.exists(target) and os.path.getmtime(target) > os.path.getmtime(src)
                and os.path.getmtime(target) > os.path.getmtime(os.path.join(HERE, launcher))
                and os.path.getmtime(target) > os.path.getmtime(os.path.join(HERE, "ref_host_shim.h"))
                and os.path.getmtime(target) > os.path.getmtime(__file__)
                and os.path.getmtime(target) > os.path.getmtime(hdr_gen)):
            continue
        cmd = ["g++", "-std=c++17", opt, "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
               "-w", "-I", HERE,
               '-DSFREF_SOURCE="%s"' % gen, os.path.join(HERE, launcher), "-o", target]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return True


def build_native(verbose=False):
    """The timed CPU build: the generated sources at -O3 -march=native for this machine's
    cores (OpenMP over the thread index).  Rebuilt whenever the machine's CPU model differs
    from the one recorded beside the libraries."""
    src_dir = os.path.join(OUT, "src")
    if not all(os.path.exists(os.path.join(src_dir, "%s.cpp" % m)) for m in MODULES):
        raise RuntimeError("oracle/_ref/src is missing: run oracle/build_ref.py where the "
                           "reference checkout is present")
    stamp = os.path.join(OUT, "native_cpu.txt")
    cpu = _cpu_model()
    fresh = os.path.exists(stamp) and open(stamp).read() == cpu
    for name, (_, launcher) in MODULES.items():
        target = lib_path(name, "_native")
        if fresh and os.path.exists(target):
            continue
        cmd = ["g++", "-std=c++17", "-O3", "-march=native", "-fPIC", "-shared", "-fopenmp", "-w",
               "-I", HERE, '-DSFREF_SOURCE="%s"' % os.path.join(src_dir, "%s.cpp" % name),
               os.path.join(HERE, launcher), "-o", target]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    with open(stamp, "w") as f:
        f.write(cpu)
    return "g++ -O3 -march=native -fopenmp (%s)" % cpu


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


if __name__ == "__main__":
    ok = build(verbose=True, opt=sys.argv[1] if len(sys.argv) > 1 else "-O2")
    sys.exit(0 if ok else 0)
