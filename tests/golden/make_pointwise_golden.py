"""Generate tests/golden/pointwise_golden.npz from the reference's own pointwise kernels.

The kernels are PyLith's libsrc/pylith/fekernels/*.hh compiled unchanged into
oracle/_ref/libref_fekernels.so (oracle/Makefile, target `ref`, which needs the
PyLith source tree). Seeded random inputs go in; the reference's outputs are
stored beside them so that the restatement (oracle/pointwise.hh) and the CUDA
pointwise code can be pinned on machines without the PyLith sources.

    python tests/golden/make_pointwise_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

NCASES = 16


def inputs(name, rng):
    s = rng.standard_normal(9)
    s_x = rng.standard_normal(18) * 1e-3
    n = rng.standard_normal(3)
    n /= np.linalg.norm(n)
    if "GenMaxwell" in name:
        a = np.concatenate([[2500.0], [3e10 * rng.uniform(0.5, 1.5)], [5e10 * rng.uniform(0.5, 1.5)],
                            rng.uniform(1.0, 10.0, 3), rng.uniform(0.1, 0.3, 3),
                            rng.standard_normal(18) * 1e-4, rng.standard_normal(6) * 1e-4])
        aoff = [0, 1, 2, 3, 6, 9, 27]
        const = [rng.uniform(0.1, 2.0)]
    elif "Fault" in name:
        a = rng.standard_normal(3)
        aoff = [0]
        const = [0.0, 0.0, 1.0, 0.5, 0.0, 0.5] if rng.random() < 0.5 else [0.0, 0.0, 1.0, 0.0, 1.0, 0.0]
    elif "bodyforce" in name:
        a = np.concatenate([[2500.0], rng.standard_normal(3)])
        aoff = [0, 1]
        const = None
    else:
        a = np.array([2500.0, 3e10 * rng.uniform(0.5, 1.5), 5e10 * rng.uniform(0.5, 1.5)])
        aoff = [0, 1, 2]
        const = None
    return s, s_x, a, aoff, const, n


def main():
    if not O.ref_available():
        O.build(ref=True)
    rng = np.random.default_rng(20261203)
    out = {}
    for name in O.KERNELS:
        key = name.replace("::", "__")
        rows = []
        for _ in range(NCASES):
            s, s_x, a, aoff, const, n = inputs(name, rng)
            numS = 2 if "Fault" in name else 1
            f = O.call_point(name, s, s_x, a, aoff, const, "ref", n=n, numS=numS)
            rows.append((s, s_x, a, np.array(aoff), np.array(const if const else [0.0]),
                         0 if const is None else len(const), n, f))
        for i, field in enumerate(["s", "s_x", "a", "aOff", "constants", "numConstants", "n", "out"]):
            out[f"{key}.{field}"] = np.array([r[i] for r in rows])
    # tangential directions, including the repeated refDir2[1] sign test (BoundaryDirections.hh:62)
    import ctypes
    lib = O.ref()
    tans = []
    for _ in range(NCASES):
        n = rng.standard_normal(3)
        n /= np.linalg.norm(n)
        r1 = np.array([0.0, 0.0, 1.0])
        r2 = rng.standard_normal(3)
        t1 = np.zeros(3)
        t2 = np.zeros(3)
        P = ctypes.c_void_p
        lib.ref_BoundaryDirections_tangential_directions(
            t1.ctypes.data_as(P), t2.ctypes.data_as(P), r1.ctypes.data_as(P), r2.ctypes.data_as(P),
            n.ctypes.data_as(P))
        tans.append(np.concatenate([n, r1, r2, t1, t2]))
    out["tangential_directions"] = np.array(tans)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pointwise_golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
