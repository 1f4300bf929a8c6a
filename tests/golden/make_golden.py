"""Writes the golden fixtures of tests/golden (run from the repository root:
``python tests/golden/make_golden.py``).

* ``recipes.json``: the error each reference test prints (tests/test_cd06.F90,
  test_cd10.F90, test_cd10_NP.F90, test_cd10_der2.F90, test_cf90.F90,
  test_filters.F90, test_filters_NP.F90, replayed as written by
  tests/recipes.py), evaluated through the oracle.
* ``oracle_small.npz``: seeded small fields and the oracle's outputs for every
  operator, both boundary kinds, every closure pair and all three axes.  The
  GPU parity tests compare the CUDA kernels with these arrays (so a GPU run
  does not depend on rebuilding the oracle identically), and the CPU tests
  check that the oracle still reproduces them bit for bit.

The Fortran reference cannot be compiled here (no Fortran compiler), so these
are outputs of the oracle, whose agreement with the reference is established
by the closed-form checks in tests/test_oracle.py.
"""
import itertools
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from tests.fields import na_nb  # noqa: E402
from tests.recipes import recipe_errors  # noqa: E402

OPS = [(oracle.CD06, oracle.D1), (oracle.CD10, oracle.D1), (oracle.CD10, oracle.D2), (oracle.CF90, oracle.FILTER)]


def cases():
    """(scheme, kind, n, dx, periodic, init bc, apply bc, axis, shape) tuples."""
    out = []
    for (scheme, kind), axis in itertools.product(OPS, (1, 2, 3)):
        n = {1: 24, 2: 12, 3: 17}[axis]
        shape = [2, 3, 2]
        shape[3 - axis] = n
        out.append(dict(scheme=scheme, kind=kind, n=n, dx=0.21, periodic=True, ibc1=0, ibcn=0, bc1=0, bcn=0,
                        axis=axis, shape=tuple(shape)))
        for bc1, bcn in itertools.product((0, 1, -1), (0, 1, -1)):
            if axis != 1 and (bc1, bcn) not in ((0, 0), (1, -1), (-1, 1)):
                continue
            ib1, ibn = (bc1, bcn) if scheme == oracle.CD06 else (0, 0)
            out.append(dict(scheme=scheme, kind=kind, n=n, dx=0.21, periodic=False, ibc1=ib1, ibcn=ibn,
                            bc1=bc1, bcn=bcn, axis=axis, shape=tuple(shape)))
    return out


def main() -> None:
    rng = np.random.default_rng(20240531)
    arrays = {}
    cs = cases()
    for i, c in enumerate(cs):
        f = rng.standard_normal(c["shape"])
        o = oracle.OracleOp(c["scheme"], c["n"], c["dx"], c["periodic"], c["ibc1"], c["ibcn"])
        na, nb = na_nb(f.shape, c["axis"])
        arrays[f"f{i}"] = f
        arrays[f"df{i}"] = o.apply(c["kind"], c["axis"], f, na, nb, c["bc1"], c["bcn"]).reshape(f.shape)
    arrays["cases"] = np.array(json.dumps(cs))
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), **arrays)
    with open(os.path.join(HERE, "recipes.json"), "w") as fh:
        json.dump(recipe_errors(), fh, indent=1, sort_keys=True)
        fh.write("\n")
    print(f"{len(cs)} cases written")


if __name__ == "__main__":
    main()
