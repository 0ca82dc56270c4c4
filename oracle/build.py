"""Build recipe for the oracle (test infrastructure only).

Two kinds of output:

* ``oracle/liboracle.so`` -- this repository's CPU restatement
  (``oracle/fold3d_oracle.c``), always built.
* ``oracle/_ref/`` -- the reference's OWN single-device code, compiled from
  the files where they lie under the reference checkout
  (``Stencil-OpenACC/AN_ISO_1_OpenACC.c`` and ``Stencil-OpenACC/Fold3dPMM.c``).
  Only generated files land in ``oracle/_ref/``:

  - ``n<N>/libref.so``: both reference translation units, ``main`` renamed
    (``-Dmain=fold3d_ref_main``), so tests can call ``ImplicitInitialiser`` and
    the six ``function_*`` sweeps directly.  Without ``-fopenacc`` the
    ``#pragma acc`` lines are ignored and ``acc_malloc``/``acc_memcpy_*``
    resolve to libgomp's host fallback, so ``T`` is a host array.
  - ``n<N>/libref_omp.so``: the same, but with the two OpenACC pragmas of each
    sweep mechanically rewritten into ``#pragma omp parallel for`` (``tnew``
    and ``F`` added to ``private``; ``:190`` omits ``tnew``).  This is a
    transform of the reference, used to time it on all host cores.
  - ``n<N>/an_iso_1_ref``: the unmodified reference program (its own
    ``main``), built only on request, used to pin the oracle against the
    reference's own text dump.

The grid size is compile-time in the reference (``Fold3dPMM.h:27-30``).  Each
build generates, in a temporary directory that is deleted afterwards, a copy
of that header with the size rewritten to N and force-includes it
(``-include``); because it defines the header's include guard, the reference
sources' own ``#include "Fold3dPMM.h"`` then expands to nothing.  The OpenMP
transform is likewise generated into the temporary directory.  Only binaries
are kept in ``oracle/_ref/``.

Flags follow the reference host build: ``-O2 -ffp-contract=off``.
The reference checkout is only needed to build ``_ref``; the built files
travel with the repository snapshot, the sources do not.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout: $FOLD3D_REFERENCE, else a directory named
# "reference" beside this checkout.
REF_ROOT = os.environ.get("FOLD3D_REFERENCE") or os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")
REF_DIR = os.path.join(REF_ROOT, "Stencil-OpenACC")
REF_OUT = os.path.join(HERE, "_ref")

CFLAGS = ["-O2", "-ffp-contract=off", "-fno-fast-math"]


def _run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def _newer(target, *deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def build_oracle(force: bool = False) -> str:
    """Compile the CPU restatement into oracle/liboracle.so."""
    src = os.path.join(HERE, "fold3d_oracle.c")
    out = os.path.join(HERE, "liboracle.so")
    if force or not _newer(out, src, __file__):
        _run(["gcc", *CFLAGS, "-fopenmp", "-fPIC", "-shared", "-Wall", "-o", out, src, "-lm"])
    return out


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REF_DIR, "AN_ISO_1_OpenACC.c"))


def _gen_header(n: int, outdir: str) -> str:
    """Reference header with the grid size of Fold3dPMM.h:27-30 set to n."""
    src = open(os.path.join(REF_DIR, "Fold3dPMM.h")).read()
    rep = {"_nx": n, "_ny": n, "_nz": n, "HEIGHT": n + 2}
    for name, val in rep.items():
        src, cnt = re.subn(r"(#define\s+%s\s+)\d+" % name, r"\g<1>%d" % val, src)
        if cnt != 1:
            raise RuntimeError("could not rewrite %s in the reference header" % name)
    path = os.path.join(outdir, "Fold3dPMM.h")
    with open(path, "w") as f:
        f.write(src)
    return path


def _omp_transform(outdir: str) -> str:
    """AN_ISO_1_OpenACC.c with each sweep's OpenACC pragmas turned into one
    OpenMP parallel-for over the same collapsed loop nest."""
    src = open(os.path.join(REF_DIR, "AN_ISO_1_OpenACC.c")).read().splitlines()
    out = []
    for line in src:
        s = line.strip()
        if s.startswith("#pragma acc parallel") or s.startswith("#pragma acc routine"):
            continue
        m = re.match(r"#pragma acc loop collapse\(2\) private\s*\((.*)\)", s)
        if m:
            names = [v.strip() for v in m.group(1).split(",") if v.strip()]
            for extra in ("tnew", "F"):
                if extra not in names:
                    names.append(extra)
            line = "#pragma omp parallel for collapse(2) schedule(static) private(%s)" % ",".join(names)
        out.append(line)
    path = os.path.join(outdir, "AN_ISO_1_omp.c")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")
    return path


def build_ref(n: int, with_program: bool = False, force: bool = False) -> str:
    """Build oracle/_ref/n<n>/{libref.so, libref_omp.so[, an_iso_1_ref]}."""
    if not reference_available():
        raise RuntimeError("reference sources not found under %s" % REF_ROOT)
    outdir = os.path.join(REF_OUT, "n%d" % n)
    os.makedirs(outdir, exist_ok=True)
    acc = os.path.join(REF_DIR, "AN_ISO_1_OpenACC.c")
    init = os.path.join(REF_DIR, "Fold3dPMM.c")
    lib = os.path.join(outdir, "libref.so")
    prog = os.path.join(outdir, "an_iso_1_ref")
    need_lib = force or not _newer(lib, acc, init, __file__)
    need_prog = with_program and (force or not _newer(prog, acc, init, __file__))
    if not (need_lib or need_prog):
        return outdir
    with tempfile.TemporaryDirectory(prefix="gen_", dir=outdir) as tmp:  # generated sources stay in _ref
        hdr = _gen_header(n, tmp)
        common = [*CFLAGS, "-w", "-include", hdr]
        if need_lib:
            _run(["gcc", *common, "-fPIC", "-shared", "-Dmain=fold3d_ref_main", "-o", lib,
                  acc, init, "-lgomp", "-lm"])
            omp_src = _omp_transform(tmp)
            _run(["gcc", *common, "-fopenmp", "-fPIC", "-shared", "-Dmain=fold3d_ref_main",
                  "-I", REF_DIR, "-o", os.path.join(outdir, "libref_omp.so"), omp_src, init,
                  "-lgomp", "-lm"])
        if need_prog:
            _run(["gcc", *common, "-o", prog, acc, init, "-lgomp", "-lm"])
    return outdir


SWEEPS = ("function_x_down", "function_x_up", "function_y_up", "function_y_down", "function_k_up",
          "function_k_down")


def dropin_path(n: int) -> str:
    return os.path.join(REF_OUT, "n%d" % n, "an_iso_1_dropin")


def build_dropin(n: int = 128, force: bool = False) -> str:
    """The reference's unmodified single-GPU program (its own main) linked
    against libfold3dpmm: its six sweep definitions are weakened in the
    object file so that the strong forwarders of
    fgcs-openacc-advanced_b200/dropin/fold3d_dropin.c take their place, and
    ImplicitInitialiser and the acc_* runtime calls resolve to the library
    (the reference's Fold3dPMM.c is not linked).  Needs libfold3dpmm.so."""
    if not reference_available():
        raise RuntimeError("reference sources not found under %s" % REF_ROOT)
    root = os.path.dirname(HERE)
    pkg = os.path.join(root, "fgcs-openacc-advanced_b200")
    lib = os.path.join(pkg, "libfold3dpmm.so")
    shim = os.path.join(pkg, "dropin", "fold3d_dropin.c")
    acc = os.path.join(REF_DIR, "AN_ISO_1_OpenACC.c")
    out = dropin_path(n)
    if not force and _newer(out, acc, lib, shim, __file__):
        return out
    if not os.path.exists(lib):
        raise RuntimeError("libfold3dpmm.so must be built first")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with tempfile.TemporaryDirectory(prefix="gen_", dir=os.path.dirname(out)) as tmp:
        hdr = _gen_header(n, tmp)
        obj = os.path.join(tmp, "an_iso_1.o")
        _run(["gcc", *CFLAGS, "-w", "-fPIC", "-fno-inline", "-include", hdr, "-c", acc, "-o", obj])
        _run(["objcopy"] + ["--weaken-symbol=%s" % s for s in SWEEPS] + [obj])
        rel = os.path.relpath(pkg, os.path.dirname(out))
        _run(["gcc", *CFLAGS, "-o", out, obj, shim, "-I", os.path.join(root, "include"), "-L", pkg,
              "-lfold3dpmm", "-Wl,-rpath,$ORIGIN/" + rel, "-lm"])
    return out


def ref_lib_path(n: int, omp: bool = False) -> str:
    return os.path.join(REF_OUT, "n%d" % n, "libref_omp.so" if omp else "libref.so")


# Sizes the tests and the CPU-baseline legs use.
DEFAULT_REF_SIZES = (8, 16, 32, 64, 128, 512, 1280)


def build_all(sizes=DEFAULT_REF_SIZES) -> None:
    """Oracle, the reference's host builds and, when libfold3dpmm.so exists,
    the reference program linked against it (build the library first)."""
    build_oracle()
    if reference_available():
        for n in sizes:
            build_ref(n)
        root = os.path.dirname(HERE)
        if os.path.exists(os.path.join(root, "fgcs-openacc-advanced_b200", "libfold3dpmm.so")):
            build_dropin(128)


if __name__ == "__main__":
    sizes = [int(a) for a in sys.argv[1:]] or list(DEFAULT_REF_SIZES)
    build_oracle()
    for n in sizes:
        print(build_ref(n, with_program=(n == 128)))
