"""ctypes binding of the CPU oracle (oracle/tortoise_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# TB_ORACLE_LIB: another build of the oracle (e.g. `make -C oracle asan`)
_LIB_PATH = os.environ.get("TB_ORACLE_LIB") or os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, dp, ip, i64 = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_int64
        L.or_create.restype = vp
        L.or_create.argtypes = [vp, C.c_int, C.c_int]
        L.or_destroy.argtypes = [vp]
        L.or_last_error.restype = C.c_char_p
        L.or_num_dofs.restype = i64
        L.or_num_dofs.argtypes = [vp]
        L.or_band_offset.restype = i64
        L.or_band_offset.argtypes = [vp, C.c_int]
        L.or_num_tuples.restype = i64
        L.or_num_tuples.argtypes = [vp, C.c_int]
        L.or_enum_counts.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64)]
        L.or_points_inside.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64), ip]
        L.or_get_tuples.argtypes = [vp, C.c_int, ip, ip]
        L.or_set_tuples.argtypes = [vp, C.c_int, i64, ip, ip]
        L.or_enumerate_items.argtypes = [vp, C.c_int, i64, i64, C.c_int]
        L.or_set_amplitude.argtypes = [vp, C.c_int, C.c_double]
        L.or_channel_propagate.argtypes = [vp, C.c_int, dp, dp, i64, i64, C.c_int, C.c_int]
        L.or_rhs.argtypes = [vp, dp, dp, C.c_int, C.c_int]
        L.or_vlasov.argtypes = [vp, C.c_int, dp, dp]
        L.or_relative_error.restype = C.c_double
        L.or_relative_error.argtypes = [vp, dp, dp]
        L.or_band_relative_error.restype = C.c_double
        L.or_band_relative_error.argtypes = [vp, C.c_int, dp, dp]
        L.or_integrate.restype = C.c_double
        L.or_integrate.argtypes = [vp, C.c_int, dp, dp]
        L.or_apply_inverse_mass.argtypes = [vp, C.c_int, dp]
        L.or_mass_matrix.argtypes = [vp, C.c_int, dp, dp]
        L.or_apply_constraints.argtypes = [vp, dp]
        L.or_dp45.restype = C.c_int
        L.or_dp45.argtypes = [vp, dp, C.c_double, C.c_double, C.c_double, dp, dp, C.c_int,
                              C.POINTER(C.c_int), C.c_int, C.c_int, i64, C.POINTER(i64), dp]
        L.or_dp45_replay.argtypes = [vp, dp, dp, i64, C.c_double, dp, C.c_int, C.c_int]
        L.or_scattering_rates.argtypes = [vp, C.c_int, C.c_int, dp, dp, C.c_int]
        L.or_set_constraint_fn.argtypes = [vp, C.c_void_p, vp]
        L.or_set_channel_amplitude_fn.restype = C.c_int
        L.or_set_channel_amplitude_fn.argtypes = [vp, C.c_int, C.c_void_p, vp]
        L.or_apply_constraints_at.restype = C.c_int
        L.or_apply_constraints_at.argtypes = [vp, dp, C.c_double]
        L.or_veto_step.restype = C.c_double
        L.or_veto_step.argtypes = [vp, C.c_double, C.c_double, C.c_double]
        L.or_gauss_constants.argtypes = [dp, dp, dp]
        L.or_veto_times.restype = C.c_double
        L.or_veto_times.argtypes = [vp, dp, C.c_int, C.c_double]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


# int fn(void* user, int32 band, double t, double* population[Ne*3])
CONSTRAINT_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_double, C.POINTER(C.c_double))


def constraint_callback(material, fn):
    """A C callback filling band b's coefficients with fn(b, t) (0 = success)."""
    sizes = [b.mesh.ne * 3 for b in material.bands]

    def cb(user, band, t, out):
        try:
            np.ctypeslib.as_array(out, shape=(sizes[band],))[:] = fn(int(band), float(t))
            return 0
        except Exception:
            return 1
    return CONSTRAINT_FN(cb)


class Oracle:
    """CPU restatement of the reference path for one material."""

    def __init__(self, material, enumerate_tuples=True, nthreads=None):
        self.material = material
        self.packed = material.pack()
        self.nthreads = nthreads or os.cpu_count() or 1
        self.h = lib().or_create(C.addressof(self.packed.desc), 1 if enumerate_tuples else 0, self.nthreads)
        if not self.h:
            raise RuntimeError("oracle: " + lib().or_last_error().decode())
        self.ndofs = lib().or_num_dofs(self.h)
        bands = material.bands
        if any(b.constrained and callable(b.constrainedPopulation) for b in bands):
            self.set_constraint(lambda b, t: bands[b].population_at(t))
        for ch, c in enumerate(material.channels):
            if getattr(c, "functAmplitude", None) is not None:
                self.set_channel_amplitude(ch, c.functAmplitude)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().or_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def band_offset(self, b):
        return lib().or_band_offset(self.h, b)

    def num_tuples(self, ch):
        return lib().or_num_tuples(self.h, ch)

    def enum_counts(self, ch):
        a, b = C.c_int64(), C.c_int64()
        lib().or_enum_counts(self.h, ch, C.byref(a), C.byref(b))
        return a.value, b.value

    def points_inside(self, ch, per_tuple=False):
        """(tuples with a Monte-Carlo point inside the simplices, such points),
        plus the count of every tuple of the list when per_tuple is set."""
        a, b = C.c_int64(), C.c_int64()
        cnt = np.zeros(self.num_tuples(ch), dtype=np.int32) if per_tuple else None
        lib().or_points_inside(self.h, ch, C.byref(a), C.byref(b), _ip(cnt) if per_tuple else None)
        return (a.value, b.value, cnt) if per_tuple else (a.value, b.value)

    def tuples(self, ch):
        n = self.num_tuples(ch)
        L = self.material.channels[ch].nlegs
        ids = np.zeros((n, L), dtype=np.int32)
        umk = np.zeros(n, dtype=np.int32)
        if n:
            lib().or_get_tuples(self.h, ch, _ip(ids), _ip(umk))
        return ids, umk

    def set_tuples(self, ch, ids, umk):
        ids = np.ascontiguousarray(ids, dtype=np.int32)
        umk = np.ascontiguousarray(umk, dtype=np.int32)
        lib().or_set_tuples(self.h, ch, umk.size, _ip(ids), _ip(umk))

    def enumerate_items(self, ch, item0, item1):
        """Channel ch's list becomes the tuples of work items [item0, item1):
        (umklapp, sections of legs 0..L-2, element choice of those legs) in
        the reference's loop order, the item index of the device's walk."""
        lib().or_enumerate_items(self.h, int(ch), int(item0), int(item1), self.nthreads)

    def set_amplitude(self, ch, a):
        lib().or_set_amplitude(self.h, ch, float(a))

    def set_constraint(self, fn):
        """Time-dependent constrained populations: fn(band, t) -> Ne*3
        coefficients for every constrained band (None: the constant ones)."""
        self._cfn = None if fn is None else constraint_callback(self.material, fn)
        lib().or_set_constraint_fn(self.h, C.cast(self._cfn, C.c_void_p) if self._cfn else None, None)

    def set_channel_amplitude(self, ch, fn):
        """functAmplitude of channel ch for its current tuple list:
        fn(barycentres[n, nlegs, 2]) -> factors[n] (None: 1)."""
        from tortoise_b200.engine import amplitude_callback
        errors = []
        cb = amplitude_callback(fn, errors) if fn is not None else None
        rc = lib().or_set_channel_amplitude_fn(self.h, ch, C.cast(cb, C.c_void_p) if cb else None, None)
        if rc != 0:
            raise errors[0] if errors else RuntimeError("oracle: " + lib().or_last_error().decode())

    def apply_constraints_at(self, f, t):
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        if lib().or_apply_constraints_at(self.h, _dp(f), float(t)) != 0:
            raise RuntimeError("oracle: " + lib().or_last_error().decode())
        return f

    def veto_step(self, t, dt, dense):
        return lib().or_veto_step(self.h, float(t), float(dt), float(dense))

    def channel_propagate(self, ch, f, t0=0, t1=-1, inverse_mass=True, out=None):
        f = np.ascontiguousarray(f, dtype=np.float64)
        if out is None:
            out = np.zeros(self.ndofs)
        lib().or_channel_propagate(self.h, ch, _dp(f), _dp(out), t0, t1, self.nthreads, 1 if inverse_mass else 0)
        return out

    def rhs(self, f, drift=True):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros(self.ndofs)
        lib().or_rhs(self.h, _dp(f), _dp(out), self.nthreads, 1 if drift else 0)
        return out

    def vlasov(self, band, fband):
        fband = np.ascontiguousarray(fband, dtype=np.float64)
        out = np.zeros_like(fband)
        lib().or_vlasov(self.h, band, _dp(fband), _dp(out))
        return out

    def relative_error(self, err, pop):
        err = np.ascontiguousarray(err, dtype=np.float64)
        pop = np.ascontiguousarray(pop, dtype=np.float64)
        return lib().or_relative_error(self.h, _dp(err), _dp(pop))

    def band_relative_error(self, band, err, pop):
        err = np.ascontiguousarray(err, dtype=np.float64)
        pop = np.ascontiguousarray(pop, dtype=np.float64)
        return lib().or_band_relative_error(self.h, band, _dp(err), _dp(pop))

    def integrate(self, band, a, b):
        a = np.ascontiguousarray(a, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        return lib().or_integrate(self.h, band, _dp(a), _dp(b))

    def mass_matrix(self, mesh=0):
        M, Mi = np.zeros(9), np.zeros(9)
        lib().or_mass_matrix(self.h, mesh, _dp(M), _dp(Mi))
        return M.reshape(3, 3), Mi.reshape(3, 3)

    def apply_constraints(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        lib().or_apply_constraints(self.h, _dp(f))
        return f

    def dp45(self, y0, t0, tf, dense, max_dense=None, drift=True, max_attempts=0):
        y = np.ascontiguousarray(y0, dtype=np.float64).copy()
        if max_dense is None:
            max_dense = int(np.ceil((tf - t0) / dense)) + 2
        dout = np.zeros((max_dense, self.ndofs))
        dt_ = np.zeros(max_dense)
        nd = C.c_int(0)
        st = (C.c_int64 * 4)()
        ds = np.zeros(3)
        rc = lib().or_dp45(self.h, _dp(y), t0, tf, dense, _dp(dout), _dp(dt_), max_dense, C.byref(nd),
                           self.nthreads, 1 if drift else 0, max_attempts, st, _dp(ds))
        n = min(nd.value, max_dense)
        return {"rc": rc, "y": y, "dense": dout[:n], "dense_t": dt_[:n], "n_dense": nd.value,
                "attempts": st[0], "accepted": st[1], "rejected": st[2], "rhs_evals": st[3],
                "t": ds[0], "dt": ds[1], "last_err": ds[2]}

    def dp45_replay(self, y0, dts, dense_s, drift=True):
        """Fixed-step Dormand-Prince over dts, then the dense output at dense_s."""
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        out = np.empty(self.ndofs)
        lib().or_dp45_replay(self.h, _dp(y0), _dp(dts), len(dts), float(dense_s), _dp(out), self.nthreads,
                             1 if drift else 0)
        return out

    def scattering_rates(self, f, ch=-1, which=-1):
        """Out-scattering rates (M^-1 applied), state-shaped; see or_scattering_rates."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty(self.ndofs)
        lib().or_scattering_rates(self.h, int(ch), int(which), _dp(f), _dp(out), self.nthreads)
        return out


def scalar_example(t0=0.0, y0=0.0, tf=10.0, dense=1.0, max_dense=64):
    """DormandPrince54.hpp:80-106 example (y' = cos t, error form 1e13 err^2)."""
    L = lib()
    L.or_dp45_scalar_example.restype = C.c_int
    L.or_dp45_scalar_example.argtypes = [C.c_double, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64)]
    d = np.zeros(max_dense)
    t = np.zeros(max_dense)
    n = C.c_int(0)
    st = (C.c_int64 * 4)()
    L.or_dp45_scalar_example(t0, y0, tf, dense, _dp(d), _dp(t), max_dense, C.byref(n), st)
    k = min(n.value, max_dense)
    return d[:k], t[:k], np.array(list(st), dtype=np.int64)
