"""CPU tests of the C-ABI: the library loads, exports every declared symbol,
and rejects bad arguments with status codes (no compute calls)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in ("fold3dpmm.h", "fold3d_acc.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = "\n".join(ln for ln in src.splitlines() if not ln.lstrip().startswith("#"))
        for m in re.finditer(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(", src):
            name = m.group(1)
            if name not in ("defined", "if", "sizeof"):
                names.add(name)
    return names


def test_every_declared_symbol_is_exported(f3d):
    decl = declared_functions()
    assert len(decl) >= 25
    out = subprocess.run(["nm", "-D", "--defined-only", f3d.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = decl - exported
    assert not missing, "declared but not exported: %s" % sorted(missing)
    assert set(f3d.EXPORTED) == decl
    # nothing else leaks from the library
    extra = {s for s in exported if not s.startswith("_")} - decl
    assert not extra, "exported but not declared: %s" % sorted(extra)


def test_version_and_default_opts(f3d):
    assert "sm_100a" in f3d.version()
    o = f3d.opts()
    assert o.max_sweeps == 1000 and o.fixed == 0 and o.tol == 0.0 and o.skip == 1


def test_null_arguments_rejected(f3d):
    L = f3d.lib()
    g = f3d.grid(8, 8, 8, 1.0)
    m = f3d.medium()
    o = f3d.opts()
    rc = L.fold3d_solve(None, C.byref(g), C.byref(m), C.c_void_p(16), C.byref(o), None, None)
    assert rc == f3d.ERR_INVALID and "ctx" in f3d.last_error()
    assert L.fold3d_create(None, 0) == f3d.ERR_INVALID


@pytest.mark.parametrize("g,msg", [((1, 8, 8, 1.0), "sizes"), ((8, 8, 8, 0.0), "spacing"),
                                   ((8, 8, 8, float("nan")), "spacing"),
                                   ((2 ** 31 - 1, 8, 8, 1.0), "too large"),
                                   ((8, 2 ** 31 - 2, 2 ** 31 - 2, 1.0), "too large"),
                                   ((70000, 70000, 70000, 1.0), "too large")])
def test_bad_grid_rejected_before_any_launch(f3d, g, msg):
    L = f3d.lib()
    gr = f3d.Grid(g[0], g[1], g[2], g[3], g[3], g[3])
    rc = L.fold3d_plane(C.byref(gr), C.byref(f3d.medium()), C.c_void_p(16), 0, 1, None)
    assert rc == f3d.ERR_INVALID and msg in f3d.last_error()


def test_bad_medium_direction_and_plane_rejected(f3d):
    L = f3d.lib()
    g = f3d.grid(8, 8, 8, 1.0)
    bad = f3d.Medium(-1.0, 0, 0, 0)
    assert L.fold3d_plane(C.byref(g), C.byref(bad), C.c_void_p(16), 0, 1, None) == f3d.ERR_INVALID
    m = f3d.medium()
    assert L.fold3d_plane(C.byref(g), C.byref(m), C.c_void_p(16), 6, 1, None) == f3d.ERR_INVALID
    assert L.fold3d_plane(C.byref(g), C.byref(m), C.c_void_p(16), 0, 8, None) == f3d.ERR_INVALID
    assert L.fold3d_plane(C.byref(g), C.byref(m), C.c_void_p(16), 1, 1, None) == f3d.ERR_INVALID
    assert L.fold3d_plane(C.byref(g), C.byref(m), None, 0, 1, None) == f3d.ERR_INVALID


def test_host_helpers_reject_bad_input(f3d):
    L = f3d.lib()
    g = f3d.grid(4, 4, 4, 1.0)
    assert L.fold3d_init_point(None, C.byref(g), 1, 1, 1) == f3d.ERR_INVALID
    import numpy as np

    T = np.zeros((6, 6, 6))
    assert L.fold3d_init_point(T.ctypes.data_as(C.c_void_p), C.byref(g), 0, 1, 1) == f3d.ERR_INVALID
    assert L.fold3d_init_point(T.ctypes.data_as(C.c_void_p), C.byref(g), 1, 1, 5) == f3d.ERR_INVALID
    assert L.fold3d_compat_set_grid(1, 5, 5) == f3d.ERR_INVALID
    assert L.fold3d_compat_set_grid(0, 0, 0) == f3d.OK


def test_create_without_gpu_fails_cleanly(f3d):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(f3d.Fold3dError) as e:
        f3d.Context(0)
    assert e.value.code in (f3d.ERR_CUDA, f3d.ERR_INVALID)


def test_oracle_library_loads(orc):
    assert orc.fold_from_point(1.1, 0, 0, 0, 1.1, 0, 0) == pytest.approx(1.0)


def test_dropin_program_links_to_library():
    """The reference's own program, linked with its sweeps replaced
    (oracle/build.py:build_dropin): the six sweeps are strong definitions
    from the forwarders, and ImplicitInitialiser and the OpenACC runtime
    calls are left to libfold3dpmm.so."""
    from oracle import build

    exe = build.dropin_path(128)
    if not os.path.exists(exe):
        pytest.skip("drop-in program not built (needs the reference sources)")
    out = subprocess.run(["nm", exe], capture_output=True, text=True, check=True).stdout
    sym = {}
    for ln in out.splitlines():
        f = ln.split()
        sym[f[-1]] = f[-2]
    for s in build.SWEEPS:
        assert sym.get(s) == "T", s
    for s in ("ImplicitInitialiser", "acc_malloc", "acc_memcpy_to_device", "acc_memcpy_from_device"):
        assert sym.get(s) == "U", s
    ldd = subprocess.run(["ldd", exe], capture_output=True, text=True).stdout
    assert "libfold3dpmm.so" in ldd and "libgomp" not in ldd


def _prototypes():
    """{name: number of parameters} of every function declared in
    include/fold3dpmm.h."""
    src = open(os.path.join(ROOT, "include", "fold3dpmm.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    src = "\n".join(ln for ln in src.splitlines() if not ln.lstrip().startswith("#"))
    out = {}
    for m in re.finditer(r"\b(\w+)\s*\(([^;{}]*?)\)\s*;", src):
        name, params = m.group(1), m.group(2).strip()
        if name in ("defined", "if", "sizeof"):
            continue
        depth, n = 0, (0 if params in ("", "void") else 1)
        for ch in params:
            depth += ch in "(["
            depth -= ch in ")]"
            n += ch == "," and depth == 0
        out[name] = n
    return out


def test_binding_argument_counts_match_header(f3d):
    """Every function the ctypes binding gives argtypes takes, in the header,
    exactly that many parameters."""
    protos = _prototypes()
    L = f3d.lib()
    checked = 0
    for name, n in protos.items():
        at = getattr(L, name).argtypes
        if at is None:
            continue
        assert len(at) == n, "%s: header %d parameters, binding %d" % (name, n, len(at))
        checked += 1
    assert checked >= 25


def test_struct_layouts_match_header(f3d, tmp_path):
    """sizeof and field offsets of the header's structs, from a C program,
    against the ctypes structures of the binding (the float32 instance
    structs share the binding's double ones: every field is a pointer)."""
    layouts = {
        "fold3d_grid": (f3d.Grid, ["nx", "ny", "nz", "dx", "dy", "dz"]),
        "fold3d_medium": (f3d.Medium, ["F", "ax", "ay", "az"]),
        "fold3d_ellip": (f3d.Ellip, ["mxx", "mxy", "mxz", "myy", "myz", "mzz"]),
        "fold3d_opts": (f3d.Opts, ["max_sweeps", "fixed", "tol", "engine", "skip", "variant"]),
        "fold3d_report": (f3d.Report, ["sweeps", "max_delta", "elapsed_ms", "nominal_updates",
                                       "evaluated_updates", "engine"]),
        "fold3d_instance": (f3d.Instance, ["grid", "medium", "T", "winners"]),
        "fold3d_instance_f32": (f3d.Instance, ["grid", "medium", "T", "winners"]),
        "fold3d_adjoint_instance": (f3d.AdjInstance, ["grid", "medium", "T", "winners", "dLdT", "lambda",
                                                      "dLdM"]),
        "fold3d_adjoint_instance_f32": (f3d.AdjInstance, ["grid", "medium", "T", "winners", "dLdT", "lambda",
                                                          "dLdM"]),
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "fold3dpmm.h"', 'int main(void) {']
    for cname, (_, fields) in layouts.items():
        lines.append('printf("%s %%zu", sizeof(%s));' % (cname, cname))
        for f in fields:
            lines.append('printf(" %%zu", offsetof(%s, %s));' % (cname, f))
        lines.append('printf("\\n");')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines():
        name, *vals = ln.split()
        got[name] = [int(v) for v in vals]
    for cname, (S, fields) in layouts.items():
        py = [C.sizeof(S)] + [getattr(S, f if f != "lambda" else "lambda_").offset for f in fields]
        assert got[cname] == py, "%s: C %s, ctypes %s" % (cname, got[cname], py)


def test_c_caller_compiles_and_links(f3d, tmp_path):
    """A C caller of the native API (tests/csrc/caller.c) compiles against
    the header and links against the library."""
    libdir = os.path.dirname(f3d.LIB_PATH)
    subprocess.run(["gcc", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "csrc", "caller.c"), "-o", str(tmp_path / "caller"), "-L", libdir,
                    "-lfold3dpmm", "-Wl,-rpath," + libdir], check=True)


def test_c_adjoint_caller_compiles(tmp_path):
    """The elliptical solve and its adjoint called from C
    (tests/csrc/gradient.c) compile against the header."""
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["gcc", "-Wall", "-Werror", "-c", "-I", os.path.join(ROOT, "include"), "-I", cuda_inc,
                    os.path.join(ROOT, "tests", "csrc", "gradient.c"), "-o", str(tmp_path / "gradient.o")],
                   check=True)


def test_newer_entry_points_reject_null_context(f3d, tmp_path):
    """Every entry point that takes a context rejects a NULL one (and NULL or
    empty instance arrays) with FOLD3D_ERR_INVALID before touching a GPU."""
    L = f3d.lib()
    g = f3d.grid(8, 8, 8, 1.0)
    e = f3d.Ellip()
    for k in ("mxx", "mxy", "mxz", "myy", "myz", "mzz"):
        setattr(e, k, 16)
    o = f3d.opts()
    rep = f3d.Report()
    p = C.c_void_p(16)  # never dereferenced: the context is checked first
    inst = (f3d.Instance * 1)()
    adj = (f3d.AdjInstance * 1)()
    calls = {
        "fold3d_solve_ellip": lambda L, s: getattr(L, s)(None, C.byref(g), C.byref(e), p, C.byref(o), None,
                                                          C.byref(rep)),
        "fold3d_solve_ellip_record": lambda L, s: getattr(L, s)(None, C.byref(g), C.byref(e), p, p, C.byref(o),
                                                                 None, C.byref(rep)),
        "fold3d_adjoint_ellip": lambda L, s: getattr(L, s)(None, C.byref(g), C.byref(e), p, p, p, p, p, 10, 0.0,
                                                            None, C.byref(rep)),
        "fold3d_solve_batch": lambda L, s: getattr(L, s)(None, 1, inst, C.byref(o), None, None),
        "fold3d_adjoint_batch": lambda L, s: getattr(L, s)(None, 1, adj, 10, 0.0, 0, None, None),
    }
    for name, call in calls.items():
        for suffix in ("", "_f32"):
            assert call(L, name + suffix) == f3d.ERR_INVALID, name + suffix
    assert L.fold3d_solve_batch(None, 0, inst, C.byref(o), None, None) == f3d.ERR_INVALID
    assert L.fold3d_solve_batch(None, 1, None, C.byref(o), None, None) == f3d.ERR_INVALID
    assert L.fold3d_adjoint_batch(None, 0, adj, 10, 0.0, 0, None, None) == f3d.ERR_INVALID
    assert L.fold3d_init_implicit_device(None, C.byref(g), C.byref(f3d.medium()), p, None) == f3d.ERR_INVALID
    T = np.zeros((10, 10, 10))
    for w in ("fold3d_write_text", "fold3d_write_raw"):
        assert getattr(L, w)(None, T.ctypes.data_as(C.c_void_p), C.byref(g)) == f3d.ERR_INVALID
    assert L.fold3d_write_vtk(None, T.ctypes.data_as(C.c_void_p), C.byref(g), 0) == f3d.ERR_INVALID


def test_binding_rejects_metric_and_batch_mismatches(f3d):
    """The Python binding checks what the C ABI cannot see behind a pointer
    before any call: a metric is six arrays with the field's shape and
    device, and a batch's lists have one entry per instance."""
    import torch

    T = torch.zeros(6, 7, 8, dtype=torch.float64)
    M = [torch.zeros(6, 7, 8, dtype=torch.float32) for _ in range(6)]
    with pytest.raises(ValueError, match="six arrays"):
        f3d.ellip(M[:5], T)
    small = [torch.zeros(4, 5, 6, dtype=torch.float32) for _ in range(6)]  # interior only: would be read past its end
    with pytest.raises(ValueError, match="field's shape"):
        f3d.ellip(small, T)
    with pytest.raises(ValueError, match="differ in length"):
        f3d.solve_batch(None, [T, T], [1.0, 1.0], [M])
    with pytest.raises(ValueError, match="differ in length"):
        f3d.solve_batch(None, [T], [1.0], [M], winners=[])
    W = torch.zeros(6, 7, 8, dtype=torch.uint8)
    with pytest.raises(ValueError, match="differ in length"):
        f3d.adjoint_batch(None, [T, T], [1.0, 1.0], [M, M], [W, W], [T, T], [T], [T, T])


def test_host_solve_rejects_a_short_output(f3d):
    """Context.solve's host path writes a whole field into `out`: a smaller
    array is refused before the library is called."""
    import numpy as np

    ctx = object.__new__(f3d.Context)  # no device needed: the check comes first
    ctx._h, ctx.device = None, 0
    T = np.zeros((6, 7, 8))
    with pytest.raises(ValueError, match="field's shape"):
        f3d.Context.solve(ctx, T, 1.0, out=np.zeros((6, 7, 7)))
    ctx._h = C.c_void_p()  # keep __del__ from closing anything


@pytest.mark.parametrize("entry", ["fold3d_solve_noalloc", "fold3d_plane"])
@pytest.mark.parametrize("bad", ["inf_spacing", "inf_F", "inf_drift", "huge_grid"])
def test_noalloc_checks_arguments_like_solve(f3d, entry, bad):
    """The allocation-free solve rejects the grids and media fold3d_solve and
    fold3d_plane reject (infinite spacing, infinite F or drift, a grid too
    large for the item counters), with the same code, before any CUDA call."""
    L = f3d.lib()
    inf = float("inf")
    g = f3d.grid(8, 8, 8, 1.0)
    m = f3d.medium()
    if bad == "inf_spacing":
        g = f3d.Grid(8, 8, 8, 1.0, inf, 1.0)
    elif bad == "inf_F":
        m = f3d.Medium(inf, 0.0, 0.0, 0.0)
    elif bad == "inf_drift":
        m = f3d.Medium(1.1, 0.0, -inf, 0.0)
    else:
        g = f3d.Grid(70000, 70000, 70000, 1.0, 1.0, 1.0)
    if entry == "fold3d_solve_noalloc":
        rc = L.fold3d_solve_noalloc(C.byref(g), C.byref(m), C.c_void_p(16), C.byref(f3d.opts(max_sweeps=2)),
                                    None, None)
    else:
        rc = L.fold3d_plane(C.byref(g), C.byref(m), C.c_void_p(16), 0, 1, None)
    assert rc == f3d.ERR_INVALID, f3d.last_error()
    assert ("spacing" in f3d.last_error()) if bad == "inf_spacing" else True
    assert ("too large" in f3d.last_error()) if bad == "huge_grid" else True
    assert ("finite" in f3d.last_error()) if bad in ("inf_F", "inf_drift") else True


def test_compat_sweep_without_grid_size_is_rejected(f3d):
    """A reference-style sweep call on a pointer that did not come from
    acc_malloc, with no grid size set, records an error and launches
    nothing."""
    L = f3d.lib()
    assert L.fold3d_compat_set_grid(0, 0, 0) == f3d.OK
    L.function_x_down(C.c_void_p(4096), 1, *([0.1] * 6), 1.1, 0.4, -0.35, 0.7)
    assert "grid size unknown" in f3d.last_error()


def test_batch_config_rejects_bad_values(f3d):
    L = f3d.lib()
    assert L.fold3d_batch_set_config(None, 4, 0) == f3d.ERR_INVALID
    a, b = C.c_int(), C.c_int()
    assert L.fold3d_batch_get_config(None, C.byref(a), C.byref(b)) == f3d.ERR_INVALID
