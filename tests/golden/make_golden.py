"""Generates the golden fixtures of tests/golden/ from the CPU oracle.

The reference ships no tests, fixtures or golden vectors for this path and
cannot be compiled here (Eigen 3.4 / oneTBB absent), so these fixtures are the
oracle's own outputs on seeded synthetic inputs.  They pin the oracle against
regressions and give the GPU parity tests fixed targets.

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

import oracle  # noqa: E402
from tortoise_b200 import workloads as W  # noqa: E402


def tuple_hash(ids, umk):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(ids, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(umk, dtype=np.int32).tobytes())
    return h.hexdigest()


def cases():
    """name -> (material builder, state seed, kT)."""
    return {
        "ee_n3": (lambda: W.parabolic_ee(3), 1, 0.1),
        "ee_n4": (lambda: W.parabolic_ee(4), 2, 0.1),
        "ee2_n3": (lambda: W.build_material(3, ("P", "D"), (), ee=True, eph=False, rtol=1e-6, atol=1e-9), 3, 0.1),
        "eph_n4": (lambda: W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0),
                                            rtol=1e-6, atol=1e-9), 4, 0.1),
        "eph_bath_n4": (lambda: W.build_material(4, ("P",), (0.15, 0.25), ee=False, eph=True, field=(0.0, 0.05),
                                                 rtol=1e-6, atol=1e-9, phonon_bath=True), 5, 0.1),
    }


def make(name):
    build, seed, kT = cases()[name]
    mat = build()
    o = oracle.Oracle(mat)
    f0 = W.initial_status(mat, kT=kT, seed=seed).vec
    out = {"f0": f0}
    for ch in range(len(mat.channels)):
        ids, umk = o.tuples(ch)
        pre, det = o.enum_counts(ch)
        out["ch%d_counts" % ch] = np.array([len(umk), pre, det], dtype=np.int64)
        out["ch%d_hash" % ch] = np.array(tuple_hash(ids, umk))
        if len(umk) <= 20000:
            out["ch%d_ids" % ch] = ids
            out["ch%d_umk" % ch] = umk
        out["ch%d_prop" % ch] = o.channel_propagate(ch, f0)
    out["rhs"] = o.rhs(f0, drift=True)
    out["rhs_nodrift"] = o.rhs(f0, drift=False)
    out["rates"] = o.scattering_rates(f0)   # MaterialStatus::scatteringRates
    for ch in range(len(mat.channels)):
        out["ch%d_rates" % ch] = o.scattering_rates(f0, ch)
    rng = np.random.default_rng(seed + 100)
    err = 1e-7 * rng.standard_normal(f0.size)
    out["err"] = err
    out["relerr"] = np.array(o.relative_error(err, f0))
    return mat, o, out


def main():
    for name in cases():
        mat, o, out = make(name)
        if name in ("eph_n4", "eph_bath_n4", "ee_n3"):
            r = o.dp45(out["f0"], 0.0, 0.4, 0.1)
            out["dp_dense"] = r["dense"]
            out["dp_dense_t"] = r["dense_t"]
            out["dp_y"] = r["y"]
            out["dp_stats"] = np.array([r["attempts"], r["accepted"], r["rejected"], r["rhs_evals"]], dtype=np.int64)
            out["dp_t"] = np.array([r["t"], r["dt"], r["last_err"]])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items() if "counts" in k})
    # reference DP54 documentation example y' = cos t
    dense, t, st = oracle.scalar_example()
    np.savez_compressed(os.path.join(HERE, "dp54_scalar.npz"), dense=dense, t=t, stats=st)


if __name__ == "__main__":
    main()
