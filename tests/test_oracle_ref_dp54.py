"""The oracle's Dormand-Prince restatement against the reference's own
integrator.

oracle/_ref/libref_dp54.so is the reference's dormandPrince54 (third overload,
include/Generics/Algorithms/DormandPrince54.hpp:479-665), compiled from the
reference tree where it lies by `make -C oracle ref` (the header needs neither
Eigen nor TBB), behind a small callback harness (oracle/ref_dp54_harness.cpp).
Each problem is integrated twice with the oracle's right-hand side,
applyConstraints(t), relativeError and timeStepVetoer plugged in, as
MaterialTimeStatus::propagate wires them (MaterialTimeStatus.cpp:102-137):
once by the reference's integrator and once by the oracle's restatement of it
(dp54_core).  Both evaluate every stage expression in the same order with
unfused operations, so they must take the same attempts and give the same
dense outputs bit for bit.  The module is skipped where the reference tree was
not there to build from.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT
from tests.golden.make_golden import cases
from tortoise_b200 import workloads as W

REF = os.path.join(ROOT, "oracle", "_ref", "libref_dp54.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref not built (no reference tree)")

DP = C.POINTER(C.c_double)
RHS = C.CFUNCTYPE(None, C.c_void_p, C.c_double, DP, DP)
ENF = C.CFUNCTYPE(None, C.c_void_p, C.c_double, DP)
NORM = C.CFUNCTYPE(C.c_double, C.c_void_p, DP, DP)
VETO = C.CFUNCTYPE(C.c_double, C.c_void_p, DP, C.c_int, C.c_double)


def _ref_lib():
    L = C.CDLL(REF)
    L.ref_dp54.restype = C.c_int64
    L.ref_dp54.argtypes = [C.c_int64, DP, C.c_double, C.c_double, C.c_double, RHS, ENF, NORM, VETO, C.c_void_p,
                           DP, DP, C.c_int64, C.POINTER(C.c_int64)]
    return L


def reference_dp54(o, y0, t0, tf, dense, drift=True, max_dense=64, rhs_fn=None):
    """The reference's integrator on the oracle's operators; rhs_fn(y) -> dy/dt
    (numpy arrays) replaces the oracle's right-hand side when given."""
    L, OL = _ref_lib(), oracle.lib()
    n = o.ndofs
    errors = []

    def rhs(user, t, y, out):
        if rhs_fn is None:
            OL.or_rhs(o.h, y, out, o.nthreads, 1 if drift else 0)
        else:
            out_np = np.ctypeslib.as_array(out, shape=(n,))
            out_np[:] = rhs_fn(np.ctypeslib.as_array(y, shape=(n,)).copy())

    def enforce(user, t, y):
        if OL.or_apply_constraints_at(o.h, y, t) != 0:
            errors.append(t)

    def norm(user, err, y):
        return OL.or_relative_error(o.h, err, y)

    def veto(user, times, ntimes, dense_step):
        return OL.or_veto_times(o.h, times, ntimes, dense_step)

    cbs = (RHS(rhs), ENF(enforce), NORM(norm), VETO(veto))
    y = np.ascontiguousarray(y0, dtype=np.float64)
    dout = np.zeros((max_dense, n))
    dt = np.zeros(max_dense)
    st = (C.c_int64 * 4)()
    nd = L.ref_dp54(n, y.ctypes.data_as(DP), t0, tf, dense, *cbs, None, dout.ctypes.data_as(DP),
                    dt.ctypes.data_as(DP), max_dense, st)
    assert not errors
    k = min(nd, max_dense)
    return {"dense": dout[:k], "dense_t": dt[:k], "n_dense": nd, "attempts": st[0], "accepted": st[1],
            "rejected": st[2], "rhs_evals": st[3]}


def _same_run(o, y0, t0, tf, dense):
    ref = reference_dp54(o, y0, t0, tf, dense)
    ours = o.dp45(y0, t0, tf, dense, max_dense=64)
    assert ours["rc"] == 0
    assert [ours["attempts"], ours["accepted"], ours["rejected"], ours["rhs_evals"]] == \
           [ref["attempts"], ref["accepted"], ref["rejected"], ref["rhs_evals"]]
    assert ours["n_dense"] == ref["n_dense"] > 0
    assert np.array_equal(ours["dense_t"], ref["dense_t"])
    assert np.array_equal(ours["dense"], ref["dense"])
    return ref


@pytest.mark.parametrize("name", ["ee_n3", "eph_n4", "eph_bath_n4"])
def test_oracle_integrator_is_the_reference_integrator(name):
    """Golden problems (one-band e-e; two-band e-ph with drift; e-ph with two
    phonon baths held by time-independent constraints)."""
    build, seed, kT = cases()[name]
    mat = build()
    f0 = W.initial_status(mat, kT=kT, seed=seed).vec
    o = oracle.Oracle(mat)
    r = _same_run(o, f0, 0.0, 0.4, 0.1)
    assert r["rejected"] >= 0 and r["attempts"] >= 4


def test_oracle_integrator_with_a_pulsed_bath():
    """A time-dependent constrained population (a bath whose temperature
    follows a Gaussian pulse): enforceValue at every stage time and the
    timeStepVetoer cutting the step before the pulse."""
    mat = W.pulsed_bath(4)
    ph = mat.bands[2]
    f0 = W.initial_status(mat, seed=2).vec
    o = oracle.Oracle(mat)
    o.set_constraint(lambda b, t: ph.population_at(t))
    pulsed = _same_run(o, f0, 0.0, 0.3, 0.01)
    o.set_constraint(lambda b, t: ph.population_at(0.0))
    flat = _same_run(o, f0, 0.0, 0.3, 0.01)
    assert pulsed["attempts"] > flat["attempts"]


def test_documentation_example_through_the_reference_integrator():
    """The scalar example of the reference's DP54 documentation
    (DormandPrince54.hpp:80-106: y' = cos t from y(0) = 0 to t = 10, dense
    step 1, normalised error 1e13 err^2) run by the reference's integrator,
    against the oracle's restatement of the same example.  The oracle carries
    t as a second state component (its core is autonomous), so the stage
    times round a little differently: same attempts, dense outputs within
    1e-12, and both within 1e-5 of sin t."""
    L = _ref_lib()
    cbs = (RHS(lambda u, t, y, out: out.__setitem__(0, np.cos(t))), ENF(lambda u, t, y: None),
           NORM(lambda u, e, y: 10000000000000. * e[0] * e[0]),
           VETO(lambda u, times, n, d: times[n - 1] - times[0]))
    y0 = np.zeros(1)
    dout, dt, st = np.zeros((64, 1)), np.zeros(64), (C.c_int64 * 4)()
    nd = L.ref_dp54(1, y0.ctypes.data_as(DP), 0.0, 10.0, 1.0, *cbs, None, dout.ctypes.data_as(DP),
                    dt.ctypes.data_as(DP), 64, st)
    d, t, stats = oracle.scalar_example(0.0, 0.0, 10.0, 1.0)
    assert nd == len(t) == 10
    assert np.array_equal(dt[:nd], t)
    assert list(stats[:3]) == [st[0], st[1], st[2]]
    assert np.max(np.abs(dout[:nd, 0] - d)) < 1e-12
    assert np.max(np.abs(dout[:nd, 0] - np.sin(dt[:nd]))) < 1e-5
