"""Regenerates the fixtures under tests/golden/ from the reference tree (run in the build container).

cases/<name>/input.dat, cases/<name>/mesh.su2.gz
    the reference's own example cases (the meshes and keyword files of its case folders), copied
    verbatim so that tests can run them where the reference tree is not mounted.
ref_<name>.npz
    outputs of the reference solver (oracle/_ref/libcsuref.so, built from the reference sources by
    oracle/Makefile) on those cases: the first residual at a fixed sample of cells and its RMS per
    variable, and the full-precision history (res[Nvar], Cx_p, Cx_v, Cy_p, Cy_v) of the first iterations.

    CSU_REFERENCE_DIR=<reference source tree> python tests/golden/make_golden.py [<reference source tree>]
"""
import gzip
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

N_ITER = 20
N_SAMPLE = 64


def copy_cases(ref_root):
    names = sorted(d for d in os.listdir(ref_root) if d.startswith("case"))
    for name in names:
        dst = os.path.join(HERE, "cases", name)
        os.makedirs(dst, exist_ok=True)
        shutil.copy(os.path.join(ref_root, name, "input.dat"), os.path.join(dst, "input.dat"))
        with open(os.path.join(ref_root, name, "mesh.su2"), "rb") as f, \
                gzip.open(os.path.join(dst, "mesh.su2.gz"), "wb", compresslevel=9) as g:
            g.write(f.read())
    return names


def make_vectors(names):
    import casekit
    from oracle.refharness import Ref
    for name in names:
        wd = casekit.materialize(name, casekit.GOLDEN_OVERRIDES.get(name, {}))
        ref = Ref(wd)
        R = ref.calc_R()
        rng = np.random.default_rng(0)
        sample = np.sort(rng.choice(ref.nc, size=min(N_SAMPLE, ref.nc), replace=False))
        ref2 = Ref(wd)
        if ref2.time_scheme == 0 and casekit.is_tube(wd):
            hist = np.zeros((0, ref2.nvar + 4))
        else:
            hist = ref2.iterate(N_ITER)
        np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), sample=sample, R_sample=R[:, sample],
                            R_rms=np.sqrt((R ** 2).mean(axis=1)), hist=hist)
        print(name, ref.nc, "cells")


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CSU_REFERENCE_DIR")
    if not ref_root:
        sys.exit("make_golden.py: name the reference source tree (argument or CSU_REFERENCE_DIR)")
    names = copy_cases(ref_root)
    make_vectors(names)
