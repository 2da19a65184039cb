"""ctypes binding of libtortoise_b200.so (include/tortoise_b200.h).

There is no CPU fallback: if the CUDA library is missing or no device is
present every call raises.
"""
import ctypes as C
import os

import numpy as np

from .abi import STATUS_NAMES

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtortoise_b200.so")

LAYOUT_AUTO, LAYOUT_MC64, LAYOUT_T64, LAYOUT_T32, LAYOUT_T40, LAYOUT_T48, LAYOUT_STREAM = 0, 1, 2, 3, 4, 5, 6
LAYOUT_NAMES = {1: "mc64", 2: "t64", 3: "t32", 4: "t40", 5: "t48", 6: "stream"}
PTR_HOST, NO_DRIFT, NO_COLLISIONS = 1, 2, 4

_lib = None


class TortoiseError(RuntimeError):
    def __init__(self, rc, where):
        self.rc = rc
        msg = lib().tb_last_error().decode(errors="replace")
        super().__init__("%s failed: %s (%s)" % (where, STATUS_NAMES.get(rc, rc), msg))


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("layout", C.c_int32), ("allow_fp32", C.c_int32),
                ("tensor_budget_bytes", C.c_int64), ("verbose", C.c_int32), ("autotune", C.c_int32),
                ("shard_rank", C.c_int32), ("shard_count", C.c_int32), ("deterministic", C.c_int32),
                ("stream_legs", C.c_int32)]


class DP45Stats(C.Structure):
    _fields_ = [("t", C.c_double), ("dt", C.c_double), ("last_err", C.c_double),
                ("attempts", C.c_int64), ("accepted", C.c_int64), ("rejected", C.c_int64),
                ("rhs_evals", C.c_int64), ("n_dense", C.c_int64), ("status", C.c_int32),
                ("done", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AdjointStats(C.Structure):
    _fields_ = [("t_obs", C.c_double), ("dense_s", C.c_double), ("steps", C.c_int64),
                ("attempts", C.c_int64), ("checkpoints", C.c_int64), ("rhs_evals", C.c_int64),
                ("vjp_evals", C.c_int64), ("status", C.c_int32), ("checkpoint_every", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib():
    """Loads the in-tree CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libtortoise_b200.so is not built: run `python -m tortoise_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, dp, ip, i64 = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.c_int64
        L.tb_last_error.restype = C.c_char_p
        L.tb_create.argtypes = [C.POINTER(vp), vp, C.POINTER(Options)]
        L.tb_destroy.argtypes = [vp]
        L.tb_num_dofs.restype = i64
        L.tb_num_dofs.argtypes = [vp]
        L.tb_band_offset.restype = i64
        L.tb_band_offset.argtypes = [vp, C.c_int]
        L.tb_num_channels.argtypes = [vp]
        L.tb_channel_info.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_int32)]
        L.tb_get_tuples.argtypes = [vp, C.c_int, ip, ip]
        L.tb_set_amplitude.argtypes = [vp, C.c_int, C.c_double]
        L.tb_rhs.argtypes = [vp, vp, vp, C.c_int]
        L.tb_channel_propagate.argtypes = [vp, C.c_int, vp, vp, C.c_int]
        L.tb_relative_error.argtypes = [vp, vp, vp, dp, C.c_int]
        L.tb_apply_constraints.argtypes = [vp, vp, C.c_int]
        L.tb_dp45_integrate.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, vp, vp, i64,
                                        C.POINTER(DP45Stats), C.c_int]
        L.tb_dp45_begin.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, i64, C.c_int]
        L.tb_dp45_advance.argtypes = [vp, i64]
        L.tb_dp45_poll.argtypes = [vp, C.POINTER(DP45Stats)]
        L.tb_dp45_end.argtypes = [vp, vp, vp, vp, i64, C.POINTER(DP45Stats), C.c_int]
        L.tb_synchronize.argtypes = [vp]
        L.tb_set_copy_wait_limit.argtypes = [vp, i64]
        L.tb_fp64_fma_rate.argtypes = [C.c_int, C.POINTER(C.c_double)]
        L.tb_get_stream.restype = vp
        L.tb_get_stream.argtypes = [vp]
        L.tb_collision_accumulate.argtypes = [vp, C.c_int, vp, vp]
        L.tb_scattering_rates.argtypes = [vp, C.c_int, C.c_int, vp, vp, C.c_int]
        L.tb_write_scatt_indices.argtypes = [vp, C.c_int, C.c_char_p]
        L.tb_read_scatt_indices.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int64),
                                            C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int64]
        L.tb_channel_schedule.argtypes = [vp, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                          C.POINTER(C.c_double)]
        L.tb_set_channel_schedule.argtypes = [vp, C.c_int, C.c_int32, C.c_int32]
        L.tb_channel_points_inside.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64)]
        L.tb_create_batch.argtypes = [C.POINTER(vp), C.POINTER(vp), C.c_int, C.POINTER(Options)]
        L.tb_num_runs.argtypes = [vp]
        L.tb_run_info.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_int32)]
        L.tb_dp45_begin_batch.argtypes = [vp, vp, dp, dp, dp, i64, C.c_int]
        L.tb_dp45_run_stats.argtypes = [vp, C.c_int, C.POINTER(DP45Stats)]
        L.tb_adjoint_rhs_vjp.argtypes = [vp, vp, vp, vp, dp, C.c_int]
        L.tb_adjoint_forward.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, C.c_int, i64, vp,
                                         C.POINTER(AdjointStats), C.c_int]
        L.tb_adjoint_backward.argtypes = [vp, vp, vp, dp, C.POINTER(AdjointStats), C.c_int]
        L.tb_adjoint_integrate.argtypes = [vp, vp, C.c_double, C.c_double, C.c_double, C.c_int, i64, vp, vp, vp,
                                           dp, C.POINTER(AdjointStats), C.c_int]
        L.tb_adjoint_steps.argtypes = [vp, dp, i64, C.POINTER(i64), dp]
        L.tb_dp45_replay.argtypes = [vp, vp, dp, i64, C.c_double, vp, C.c_int]
        L.tb_set_constraint_fn.argtypes = [vp, C.c_void_p, vp]
        L.tb_set_channel_amplitude_fn.argtypes = [vp, C.c_int, C.c_void_p, vp]
        L.tb_apply_constraints_at.argtypes = [vp, vp, C.c_double, C.c_int]
        L.tb_shard_range.argtypes = [i64, C.c_int, C.c_int, C.POINTER(i64), C.POINTER(i64)]
        L.tb_shard_unique_id.argtypes = [C.c_char_p]
        L.tb_shard_connect.argtypes = [vp, C.c_char_p, C.c_double]
        L.tb_shard_info.argtypes = [vp, C.c_int, C.POINTER(i64), C.POINTER(i64)]
        _lib = L
    return _lib


def _check(rc, where):
    if rc != 0:
        raise TortoiseError(rc, where)


def _hp(a):
    return C.c_void_p(a.ctypes.data)


SHARD_ID_BYTES = 128

# tb_constraint_fn: int fn(void* user, int32 band, double t, double* population)
CONSTRAINT_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_double, C.POINTER(C.c_double))
# tb_amplitude_fn: int fn(void* user, int64 n, int32 nlegs, const double* barycentres, double* out)
AMPLITUDE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double))


def amplitude_callback(fn, errors):
    """A tb_amplitude_fn calling fn(barycentres[n, nlegs, 2]) -> factors[n]."""
    def cb(user, n, nlegs, bary, out):
        try:
            b = np.ctypeslib.as_array(bary, shape=(int(n), int(nlegs), 2))
            np.ctypeslib.as_array(out, shape=(int(n),))[:] = fn(b)
            return 0
        except Exception as exc:
            errors.append(exc)
            return 1
    return AMPLITUDE_FN(cb)


def shard_range(n_tuples, rank, n_ranks):
    """[begin, end) of the tuples that rank ``rank`` of ``n_ranks`` keeps
    (tb_shard_range; host arithmetic, no device needed)."""
    b, e = C.c_int64(), C.c_int64()
    _check(lib().tb_shard_range(int(n_tuples), int(rank), int(n_ranks), C.byref(b), C.byref(e)), "tb_shard_range")
    return b.value, e.value


def fp64_fma_rate(device=0):
    """The device's measured FP64 FMA throughput, FMAs per second (tb_fp64_fma_rate)."""
    v = C.c_double()
    _check(lib().tb_fp64_fma_rate(int(device), C.byref(v)), "tb_fp64_fma_rate")
    return v.value


def shard_unique_id():
    """A new communicator id (bytes) for tb_shard_connect; one rank makes it."""
    buf = C.create_string_buffer(SHARD_ID_BYTES)
    _check(lib().tb_shard_unique_id(buf), "tb_shard_unique_id")
    return buf.raw


def _shard_opts(shard):
    if shard is None:
        return 0, 0
    rank, count = shard
    return int(rank), int(count)


class Engine:
    """One device handle for a Material (tb_create ... tb_destroy).

    shard=(rank, count): this process keeps the rank-th part of every tuple
    list (one GPU per rank); connect the ranks with ``shard_connect`` (or
    tortoise_b200.shard.connect) so that collision sums are all-reduced.

    deterministic=True: bit-reproducible sums (tb_options.deterministic):
    exact fixed-point accumulation instead of FP64 atomics.

    stream_legs=L (2..4): channels with at least L legs keep no tuple list
    and enumerate their tuples in every evaluation (tb_options.stream_legs)."""

    def __init__(self, material, layout=LAYOUT_AUTO, allow_fp32=False, device=0, tensor_budget_bytes=0,
                 autotune=False, shard=None, deterministic=False, stream_legs=0):
        self.material = material
        self.packed = material.pack()
        opts = Options(device, layout, int(allow_fp32), tensor_budget_bytes, 0, int(autotune), *_shard_opts(shard),
                       int(bool(deterministic)), int(stream_legs))
        h = C.c_void_p()
        _check(lib().tb_create(C.byref(h), C.addressof(self.packed.desc), C.byref(opts)), "tb_create")
        self.h = h
        self.ndofs = lib().tb_num_dofs(h)
        self._install_constraints()

    def _bands(self):
        return list(self.material.bands)

    def _channels(self):
        return list(self.material.channels)

    def _install_constraints(self):
        """Bands whose constrainedPopulation is a callable of time get it as
        the handle's constraint callback; channels with a functAmplitude get
        their per-tuple factors."""
        bands = self._bands()
        if any(b.constrained and callable(b.constrainedPopulation) for b in bands):
            self.set_constraint(lambda b, t: bands[b].population_at(t))
        for ch, c in enumerate(self._channels()):
            if getattr(c, "functAmplitude", None) is not None:
                self.set_channel_amplitude(ch, c.functAmplitude)

    def set_channel_amplitude(self, ch, fn):
        """ScatteringChannel::functAmplitude (tb_set_channel_amplitude_fn):
        fn(barycentres[n, nlegs, 2]) -> factors[n], evaluated once per tuple at
        its elements' barycentres; None returns to 1.  In a batch the factors
        belong to the channel's structure group."""
        errors = []
        cb = amplitude_callback(fn, errors) if fn is not None else None
        rc = lib().tb_set_channel_amplitude_fn(self.h, ch, C.cast(cb, C.c_void_p) if cb else None, None)
        if rc != 0 and errors:
            raise errors[0]
        _check(rc, "tb_set_channel_amplitude_fn")

    def set_constraint(self, fn):
        """Time-dependent constrained populations (tb_set_constraint_fn):
        fn(band, t) -> Ne*3 coefficients of constrained band `band` (global
        index) at time t; None returns to the description's constant ones."""
        if fn is None:
            self._cfn = None
            _check(lib().tb_set_constraint_fn(self.h, None, None), "tb_set_constraint_fn")
            return
        sizes = [b.mesh.ne * 3 for b in self._bands()]
        self.constraint_error = None

        def cb(user, band, t, out):
            try:
                np.ctypeslib.as_array(out, shape=(sizes[band],))[:] = fn(int(band), float(t))
                return 0
            except Exception as exc:   # reported as TB_ERR_ARG by the library
                self.constraint_error = exc
                return 1
        self._cfn = CONSTRAINT_FN(cb)
        _check(lib().tb_set_constraint_fn(self.h, C.cast(self._cfn, C.c_void_p), None), "tb_set_constraint_fn")

    def apply_constraints_at(self, f, t):
        """MaterialStatus::applyConstraints(t) on a host state (returns a copy)."""
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        _check(lib().tb_apply_constraints_at(self.h, _hp(f), float(t), PTR_HOST), "tb_apply_constraints_at")
        return f

    def close(self):
        if getattr(self, "h", None):
            lib().tb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- introspection --------------------------------------------------
    def channel_info(self, ch):
        n, p, d = C.c_int64(), C.c_int64(), C.c_int64()
        lay = C.c_int32()
        _check(lib().tb_channel_info(self.h, ch, C.byref(n), C.byref(p), C.byref(d), C.byref(lay)), "tb_channel_info")
        return {"n_tuples": n.value, "n_prefilter": p.value, "n_det": d.value, "layout": LAYOUT_NAMES.get(lay.value)}

    def points_inside(self, ch):
        """(tuples with a Monte-Carlo point inside the simplices, such points),
        or (-1, -1) when the channel has no such list."""
        n, p = C.c_int64(), C.c_int64()
        _check(lib().tb_channel_points_inside(self.h, ch, C.byref(n), C.byref(p)), "tb_channel_points_inside")
        return n.value, p.value

    def write_scatt_indices(self, ch, path):
        """The channel's tuple list in the reference's .scattIndices format."""
        _check(lib().tb_write_scatt_indices(self.h, ch, os.fsencode(path)), "tb_write_scatt_indices")

    def shard_info(self, ch):
        """(index of this handle's first tuple in the full list, full list length)."""
        b, n = C.c_int64(), C.c_int64()
        _check(lib().tb_shard_info(self.h, ch, C.byref(b), C.byref(n)), "tb_shard_info")
        return b.value, n.value

    def shard_connect(self, unique_id, timeout_s=60.0):
        """Joins this handle to the communicator ``unique_id`` (tb_shard_connect);
        every rank calls it with the same id."""
        if len(unique_id) != SHARD_ID_BYTES:
            raise ValueError("a shard id has %d bytes" % SHARD_ID_BYTES)
        _check(lib().tb_shard_connect(self.h, bytes(unique_id), float(timeout_s)), "tb_shard_connect")

    def set_schedule(self, ch, stages, pair=0, runs=0, inside_only=None):
        """Pins the contraction schedule of channel ch's group (tb_set_channel_schedule):
        runs = 32, 16, 8 or 4 selects the run-minor contraction, else pair = 0 or 1.
        Monte-Carlo channels: stages 0 and inside_only = True (only the points
        inside the simplices) or False (every point of every tuple)."""
        if inside_only is not None:
            code = 6 if inside_only else 0
        else:
            code = {32: 2, 8: 3, 4: 4, 16: 5}[runs] if runs else int(pair)
        _check(lib().tb_set_channel_schedule(self.h, ch, int(stages), code), "tb_set_channel_schedule")

    def schedule(self, ch):
        st, pr, sec = C.c_int32(), C.c_int32(), C.c_double()
        _check(lib().tb_channel_schedule(self.h, ch, C.byref(st), C.byref(pr), C.byref(sec)), "tb_channel_schedule")
        # runs: run-minor lane-group width (32, 16, 8 or 4 runs per tuple), 0 = off
        d = {"stages": st.value, "pair": int(pr.value == 1), "runs": {2: 32, 3: 8, 4: 4, 5: 16}.get(pr.value, 0),
             "tuned_seconds": sec.value}
        if pr.value == 6:   # Monte-Carlo channel visiting only the points inside the simplices
            d["inside_only"] = True
        if pr.value == 7:   # streamed channel: tuples enumerated in every evaluation
            d["inside_only"] = True
            d["streamed"] = True
        return d

    def tuples(self, ch):
        info = self.channel_info(ch)
        L = self.material.channels[ch].nlegs
        ids = np.zeros((info["n_tuples"], L), dtype=np.int32)
        umk = np.zeros(info["n_tuples"], dtype=np.int32)
        _check(lib().tb_get_tuples(self.h, ch, ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                   umk.ctypes.data_as(C.POINTER(C.c_int32))), "tb_get_tuples")
        return ids, umk

    def set_amplitude(self, ch, a):
        _check(lib().tb_set_amplitude(self.h, ch, float(a)), "tb_set_amplitude")

    def set_copy_wait_limit(self, polls):
        """Poll limit of the contraction kernels' wait for staged moment tiles
        (tb_set_copy_wait_limit; 0 gives up at once)."""
        _check(lib().tb_set_copy_wait_limit(self.h, int(polls)), "tb_set_copy_wait_limit")

    # -- host-pointer calls ----------------------------------------------
    def rhs(self, f, drift=True, collisions=True):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty(self.ndofs)
        flags = PTR_HOST | (0 if drift else NO_DRIFT) | (0 if collisions else NO_COLLISIONS)
        _check(lib().tb_rhs(self.h, _hp(f), _hp(out), flags), "tb_rhs")
        return out

    def channel_propagate(self, ch, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty(self.ndofs)
        _check(lib().tb_channel_propagate(self.h, ch, _hp(f), _hp(out), PTR_HOST), "tb_channel_propagate")
        return out

    def scattering_rates(self, f, ch=-1, leg=-1):
        """Out-scattering rates (MaterialStatus::scatteringRates for ch = leg = -1)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty(self.ndofs)
        _check(lib().tb_scattering_rates(self.h, int(ch), int(leg), _hp(f), _hp(out), PTR_HOST), "tb_scattering_rates")
        return out

    def relative_error(self, err, pop):
        err = np.ascontiguousarray(err, dtype=np.float64)
        pop = np.ascontiguousarray(pop, dtype=np.float64)
        r = np.zeros(max(1, lib().tb_num_runs(self.h)))
        _check(lib().tb_relative_error(self.h, _hp(err), _hp(pop), r.ctypes.data_as(C.POINTER(C.c_double)),
                                       PTR_HOST), "tb_relative_error")
        return float(r[0]) if r.size == 1 else r

    def apply_constraints(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        _check(lib().tb_apply_constraints(self.h, _hp(f), PTR_HOST), "tb_apply_constraints")
        return f

    def dp45(self, y0, t0, tf, dense, max_dense=None, drift=True):
        y = np.ascontiguousarray(y0, dtype=np.float64).copy()
        if max_dense is None:
            max_dense = int(np.ceil((tf - t0) / dense)) + 2
        dout = np.zeros((max(max_dense, 1), self.ndofs))
        dt_ = np.zeros(max(max_dense, 1))
        st = DP45Stats()
        flags = PTR_HOST | (0 if drift else NO_DRIFT)
        rc = lib().tb_dp45_integrate(self.h, _hp(y), t0, tf, dense, _hp(dout), _hp(dt_), max_dense, C.byref(st), flags)
        n = min(st.n_dense, max_dense)
        res = st.as_dict()
        res.update({"rc": rc, "y": y, "dense": dout[:n], "dense_t": dt_[:n]})
        return res

    # -- device-pointer calls (torch tensors or raw addresses) --------------
    def rhs_device(self, f_ptr, out_ptr, flags=0):
        _check(lib().tb_rhs(self.h, C.c_void_p(f_ptr), C.c_void_p(out_ptr), flags), "tb_rhs")

    def dp45_begin(self, y0, t0, tf, dense, max_dense=0, drift=True):
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        flags = PTR_HOST | (0 if drift else NO_DRIFT)
        _check(lib().tb_dp45_begin(self.h, _hp(y0), t0, tf, dense, max_dense, flags), "tb_dp45_begin")

    def dp45_advance(self, n):
        _check(lib().tb_dp45_advance(self.h, int(n)), "tb_dp45_advance")

    def dp45_poll(self):
        st = DP45Stats()
        _check(lib().tb_dp45_poll(self.h, C.byref(st)), "tb_dp45_poll")
        return st.as_dict()

    def channel_count(self):
        return lib().tb_num_channels(self.h)

    def stream_ptr(self):
        return lib().tb_get_stream(self.h)

    def collision_accumulate(self, f_ptr, acc_ptr, ch=-1):
        _check(lib().tb_collision_accumulate(self.h, ch, C.c_void_p(f_ptr), C.c_void_p(acc_ptr)),
               "tb_collision_accumulate")

    def synchronize(self):
        _check(lib().tb_synchronize(self.h), "tb_synchronize")

    # -- adjoint -------------------------------------------------------------
    def rhs_vjp(self, f, theta, drift=True, collisions=True):
        """(dF/df)^T theta and dF/d amplitude_c . theta per channel (host arrays)."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        theta = np.ascontiguousarray(theta, dtype=np.float64)
        g = np.empty(self.ndofs)
        ga = np.zeros(max(1, self.channel_count()))
        flags = PTR_HOST | (0 if drift else NO_DRIFT) | (0 if collisions else NO_COLLISIONS)
        _check(lib().tb_adjoint_rhs_vjp(self.h, _hp(f), _hp(theta), _hp(g), ga.ctypes.data_as(C.POINTER(C.c_double)),
                                        flags), "tb_adjoint_rhs_vjp")
        return g, ga[:self.channel_count()]

    def adjoint_forward(self, y0, t0, tf, dense, checkpoint_every=16, max_steps=16384, drift=True):
        """Differentiable forward sweep; returns f at the last dense output and stats."""
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        fo = np.empty(self.ndofs)
        st = AdjointStats()
        flags = PTR_HOST | (0 if drift else NO_DRIFT)
        _check(lib().tb_adjoint_forward(self.h, _hp(y0), t0, tf, dense, int(checkpoint_every), int(max_steps),
                                        _hp(fo), C.byref(st), flags), "tb_adjoint_forward")
        return fo, st.as_dict()

    def adjoint_backward(self, lam):
        """Gradients of <lam, f(t_obs)> wrt f0 and the channel amplitudes."""
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        g = np.empty(self.ndofs)
        ga = np.zeros(max(1, self.channel_count()))
        st = AdjointStats()
        _check(lib().tb_adjoint_backward(self.h, _hp(lam), _hp(g), ga.ctypes.data_as(C.POINTER(C.c_double)),
                                         C.byref(st), PTR_HOST), "tb_adjoint_backward")
        return g, ga[:self.channel_count()], st.as_dict()

    def adjoint_steps(self):
        n, s = C.c_int64(), C.c_double()
        _check(lib().tb_adjoint_steps(self.h, None, 0, C.byref(n), C.byref(s)), "tb_adjoint_steps")
        dts = np.zeros(max(1, n.value))
        _check(lib().tb_adjoint_steps(self.h, dts.ctypes.data_as(C.POINTER(C.c_double)), n.value, C.byref(n),
                                      C.byref(s)), "tb_adjoint_steps")
        return dts[:n.value], s.value

    def dp45_replay(self, y0, dts, dense_s, drift=True):
        """Fixed-step Dormand-Prince over dts, then the dense output at dense_s."""
        y0 = np.ascontiguousarray(y0, dtype=np.float64)
        dts = np.ascontiguousarray(dts, dtype=np.float64)
        out = np.empty(self.ndofs)
        flags = PTR_HOST | (0 if drift else NO_DRIFT)
        _check(lib().tb_dp45_replay(self.h, _hp(y0), dts.ctypes.data_as(C.POINTER(C.c_double)), len(dts),
                                    float(dense_s), _hp(out), flags), "tb_dp45_replay")
        return out


class BatchEngine(Engine):
    """Several independent runs (Materials) in one device handle
    (tb_create_batch).  Runs with identical structure share tuple lists and
    moment tensors; each keeps its own amplitudes, tolerances, state and step
    size.  Channels and bands are numbered globally in run order."""

    def __init__(self, materials, layout=LAYOUT_AUTO, allow_fp32=False, device=0, tensor_budget_bytes=0,
                 autotune=False, shard=None, deterministic=False, stream_legs=0):
        self.materials = list(materials)
        self.material = self.materials[0]
        self.packs = [m.pack() for m in self.materials]
        arr = (C.c_void_p * len(self.packs))(*[C.addressof(p.desc) for p in self.packs])
        opts = Options(device, layout, int(allow_fp32), tensor_budget_bytes, 0, int(autotune), *_shard_opts(shard),
                       int(bool(deterministic)), int(stream_legs))
        h = C.c_void_p()
        _check(lib().tb_create_batch(C.byref(h), arr, len(self.packs), C.byref(opts)), "tb_create_batch")
        self.h = h
        self.ndofs = lib().tb_num_dofs(h)
        self.nruns = len(self.packs)
        self._install_constraints()
        self.slices, self.chan0 = [], []
        for r in range(self.nruns):
            off, n = C.c_int64(), C.c_int64()
            b0, c0 = C.c_int32(), C.c_int32()
            _check(lib().tb_run_info(h, r, C.byref(off), C.byref(n), C.byref(b0), C.byref(c0)), "tb_run_info")
            self.slices.append(slice(off.value, off.value + n.value))
            self.chan0.append(c0.value)

    def _bands(self):
        return [b for m in self.materials for b in m.bands]

    def _channels(self):
        return [c for m in self.materials for c in m.channels]

    def tuples(self, ch):
        r = max(i for i in range(self.nruns) if self.chan0[i] <= ch)
        info = self.channel_info(ch)
        L = self.materials[r].channels[ch - self.chan0[r]].nlegs
        ids = np.zeros((info["n_tuples"], L), dtype=np.int32)
        umk = np.zeros(info["n_tuples"], dtype=np.int32)
        _check(lib().tb_get_tuples(self.h, ch, ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                   umk.ctypes.data_as(C.POINTER(C.c_int32))), "tb_get_tuples")
        return ids, umk

    def run_stats(self, r):
        """Run r's integration counters as of the last dp45_poll (tb_dp45_run_stats)."""
        rs = DP45Stats()
        _check(lib().tb_dp45_run_stats(self.h, int(r), C.byref(rs)), "tb_dp45_run_stats")
        return rs.as_dict()

    def split(self, vec):
        return [np.asarray(vec)[s] for s in self.slices]

    def dp45(self, y0, t0, tf, dense, max_dense=None, drift=True):
        """Integrates every run; t0, tf, dense may be scalars or per-run lists."""
        y = np.ascontiguousarray(y0, dtype=np.float64).copy()
        as_arr = lambda x: np.ascontiguousarray(np.broadcast_to(np.asarray(x, dtype=np.float64), (self.nruns,)))
        t0a, tfa, da = as_arr(t0), as_arr(tf), as_arr(dense)
        if max_dense is None:
            max_dense = int(np.ceil(np.max((tfa - t0a) / da))) + 2
        flags = PTR_HOST | (0 if drift else NO_DRIFT)
        dp = C.POINTER(C.c_double)
        _check(lib().tb_dp45_begin_batch(self.h, _hp(y), t0a.ctypes.data_as(dp), tfa.ctypes.data_as(dp),
                                         da.ctypes.data_as(dp), max_dense, flags), "tb_dp45_begin_batch")
        batch = 4
        while True:
            self.dp45_advance(batch)
            if self.dp45_poll()["done"]:
                break
            batch = min(64, batch * 2)
        sizes = [s.stop - s.start for s in self.slices]
        dout = np.zeros(max_dense * sum(sizes))
        dts = np.zeros(max_dense * self.nruns)
        st = DP45Stats()
        rc = lib().tb_dp45_end(self.h, _hp(y), _hp(dout), _hp(dts), max_dense, C.byref(st), PTR_HOST)
        runs, off = [], 0
        for r in range(self.nruns):
            rs = DP45Stats()
            _check(lib().tb_dp45_run_stats(self.h, r, C.byref(rs)), "tb_dp45_run_stats")
            d = rs.as_dict()
            nd = min(rs.n_dense, max_dense)
            d["dense"] = dout[off:off + max_dense * sizes[r]].reshape(max_dense, sizes[r])[:nd]
            d["dense_t"] = dts[r * max_dense:r * max_dense + nd]
            d["y"] = y[self.slices[r]]
            runs.append(d)
            off += max_dense * sizes[r]
        return {"rc": rc, "y": y, "runs": runs}
