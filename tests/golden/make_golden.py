"""Generate tests/golden/ from the reference's OWN code.

Run in a checkout where the reference sources are available; it builds
oracle/_ref (oracle/build.py compiles Stencil-OpenACC/AN_ISO_1_OpenACC.c and
Stencil-OpenACC/Fold3dPMM.c for the host at each size) and drives the
reference's ImplicitInitialiser and six function_* sweeps in the order and
with the arguments of its main (AN_ISO_1_OpenACC.c:1180-1237).

Outputs:
  ref_n8.npz, ref_n16.npz   full fields (float64, shape (n+2,)*3):
      init            after ImplicitInitialiser
      s1, s2, s8      after 1, 2 and 8 sweeps (implicit-surface source)
      point_s8        point source at the centre (+MAXT elsewhere), 8 sweeps
  digests.json      sha256 of the raw float64 bytes of larger reference
                    results (the fields themselves would be too big): at 32,
                    37, 64 and 99 the initial field, 8 sweeps from it and 8
                    sweeps from a centred point source; at 37 and 99 also 8
                    sweeps from point sources next to a corner and on a face.
                    Plus the md5 of the reference program's own text dump at
                    128^3 (an_iso_1_openacc.txt, written by its unmodified
                    main).

  digests_large.json  sha256 digests at the benchmarked sizes, from the
                    OpenMP transform of the reference (libref_omp.so, the same
                    arithmetic in the same order per point; a plane's points
                    are independent, so the result is the same bits, which
                    tests/test_oracle.py checks against libref.so):
                      n512_init, n512_s8      implicit surface, 8 sweeps
                      n512_point_s8           point source at (i,j,k) =
                                              (65, 257, 257), 8 sweeps
                      n1280_init, n1280_s1 .. implicit surface after 1, 2,
                                              ... sweeps, as far as --sweeps1280
                    Written after every result, so an interrupted run keeps
                    what it finished.

    python tests/golden/make_golden.py            # everything but 128^3 dump
    python tests/golden/make_golden.py --dump128  # also run the 128^3 program (~30 s)
    python tests/golden/make_golden.py --large [--sweeps1280 K]
        # only digests_large.json: 512^3 (~20 min on 8 cores) and 1280^3
        # (34 GB of host memory; init ~10 min, ~20 min per sweep on 8 cores)
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import MAXT, RefLib, build  # noqa: E402


def point_field(n, src=None):
    """MAXT everywhere, 0 at src = (i, j, k) (1-based; default the centre)."""
    T = np.full((n + 2,) * 3, MAXT)
    i, j, k = src if src is not None else (n // 2 + 1,) * 3
    T[k, j, i] = 0.0
    return T


# off-centre point sources (1-based i, j, k) for the digests of n = 37 and 99
OFF_CENTRE = {
    "corner_point": lambda n: (2, 1, 2),
    "face_point": lambda n: (n, n // 3 + 1, 2 * n // 3 + 1),
}


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


# point source of the 512^3 digest (1-based i, j, k; x fastest)
POINT_512 = (65, 257, 257)


def main_large(sweeps1280: int) -> None:
    path = os.path.join(HERE, "digests_large.json")
    dig = json.load(open(path)) if os.path.exists(path) else {}

    def put(key, T):
        dig[key] = sha(T)
        with open(path, "w") as fh:
            json.dump(dig, fh, indent=1, sort_keys=True)
        print(key, dig[key], flush=True)

    build.build_ref(512)
    r = RefLib(512, omp=True)
    if "n512_s8" not in dig:
        T = r.init_implicit()
        put("n512_init", T)
        r.sweeps(T, 8)
        put("n512_s8", T)
        del T
    if "n512_point_s8" not in dig:
        P = point_field(512, POINT_512)
        r.sweeps(P, 8)
        put("n512_point_s8", P)
        del P
    if sweeps1280 > 0:
        build.build_ref(1280)
        r = RefLib(1280, omp=True)
        T = r.init_implicit()
        put("n1280_init", T)
        for s in range(1, sweeps1280 + 1):
            r.sweeps(T, 1)
            put("n1280_s%d" % s, T)


def main():
    if "--large" in sys.argv:
        k = sys.argv.index("--sweeps1280") + 1 if "--sweeps1280" in sys.argv else 0
        main_large(int(sys.argv[k]) if k else 1)
        return
    out = {}
    for n in (8, 16):
        build.build_ref(n)
        r = RefLib(n)
        T = r.init_implicit()
        f = {"init": T.copy()}
        r.sweeps(T, 1)
        f["s1"] = T.copy()
        r.sweeps(T, 1)
        f["s2"] = T.copy()
        r.sweeps(T, 6)
        f["s8"] = T.copy()
        P = point_field(n)
        r.sweeps(P, 8)
        f["point_s8"] = P
        np.savez_compressed(os.path.join(HERE, "ref_n%d.npz" % n), **f)
    dig = {}
    for n in (32, 37, 64, 99):  # 37 and 99: sizes that leave partial tiles on every axis
        build.build_ref(n)
        r = RefLib(n)
        T = r.init_implicit()
        dig["n%d_init" % n] = sha(T)
        r.sweeps(T, 8)
        dig["n%d_s8" % n] = sha(T)
        P = point_field(n)
        r.sweeps(P, 8)
        dig["n%d_point_s8" % n] = sha(P)
        if n in (37, 99):  # sources next to a corner and on a face
            for name, src in OFF_CENTRE.items():
                P = point_field(n, src(n))
                r.sweeps(P, 8)
                dig["n%d_%s_s8" % (n, name)] = sha(P)
    if "--dump128" in sys.argv:
        d = build.build_ref(128, with_program=True)
        with tempfile.TemporaryDirectory(prefix="run_", dir=d) as tmp:
            subprocess.run([os.path.join(d, "an_iso_1_ref")], cwd=tmp, check=True,
                           stdout=subprocess.DEVNULL)
            with open(os.path.join(tmp, "an_iso_1_openacc.txt"), "rb") as fh:
                dig["n128_s8_text_md5"] = hashlib.md5(fh.read()).hexdigest()
    else:
        old = os.path.join(HERE, "digests.json")
        if os.path.exists(old):
            prev = json.load(open(old))
            if "n128_s8_text_md5" in prev:
                dig["n128_s8_text_md5"] = prev["n128_s8_text_md5"]
    with open(os.path.join(HERE, "digests.json"), "w") as fh:
        json.dump(dig, fh, indent=1, sort_keys=True)
    print(json.dumps(dig, indent=1))


if __name__ == "__main__":
    main()
