"""ctypes mirror of include/tortoise_b200.h (the problem description structs).

Only data layout lives here; the entry points are bound in
``tortoise_b200.engine``.  The structs must stay byte-identical to the C header.
"""
import ctypes as C

import numpy as np

TB_MAX_LEGS = 4
IN, OUT = 1, -1
FERMION, BOSON = -1, 1

STATUS_NAMES = {
    0: "TB_OK", 1: "TB_ERR_BAD_DESC", 2: "TB_ERR_OOM", 3: "TB_ERR_CUDA",
    4: "TB_ERR_DT_UNDERFLOW", 5: "TB_ERR_NONFINITE", 6: "TB_ERR_TIMEOUT",
    7: "TB_ERR_NO_DEVICE", 8: "TB_ERR_ARG", 9: "TB_ERR_CAPACITY",
}

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class TbRegion(C.Structure):
    _fields_ = [("origin", C.c_double * 2), ("gvec", C.c_double * 4)]


class TbMeshDesc(C.Structure):
    _fields_ = [("rel_origin", C.c_double * 2), ("rel_size", C.c_double * 2),
                ("nsplit", C.c_int32 * 2)]


class TbBandDesc(C.Structure):
    _fields_ = [("mesh", C.c_int32), ("charge", C.c_double), ("statistics", C.c_double),
                ("dispersion", _dp), ("abs_tol", C.c_double), ("rel_tol", C.c_double),
                ("penalisation", C.c_double), ("constrained", C.c_int32),
                ("constrained_population", _dp), ("drift_velocity", C.c_double * 2)]


class TbChannelDesc(C.Structure):
    _fields_ = [("nlegs", C.c_int32), ("band", C.c_int32 * TB_MAX_LEGS),
                ("dir", C.c_int32 * TB_MAX_LEGS), ("amplitude", C.c_double),
                ("n_mc", C.c_int32), ("min_det", C.c_double), ("threshold", C.c_double),
                ("n_umklapp", C.c_int32), ("umklapp", _dp), ("mc_points", _dp),
                ("mc_points_precalc", _dp), ("n_tuples", C.c_int64), ("tuples", _ip),
                ("tuple_umklapp", _ip)]


class TbProblemDesc(C.Structure):
    _fields_ = [("region", TbRegion), ("n_meshes", C.c_int32),
                ("meshes", C.POINTER(TbMeshDesc)), ("n_bands", C.c_int32),
                ("bands", C.POINTER(TbBandDesc)), ("n_channels", C.c_int32),
                ("channels", C.POINTER(TbChannelDesc))]


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array (None -> NULL)."""
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_ip)


class PackedProblem:
    """Owns the numpy buffers behind a TbProblemDesc so the pointers stay valid."""

    def __init__(self, region, meshes, bands, channels):
        self._keep = []
        d = TbProblemDesc()
        d.region.origin[:] = [float(x) for x in region.origin]
        d.region.gvec[:] = [float(region.gvec[0, 0]), float(region.gvec[1, 0]),
                            float(region.gvec[0, 1]), float(region.gvec[1, 1])]
        marr = (TbMeshDesc * max(1, len(meshes)))()
        for i, m in enumerate(meshes):
            marr[i].rel_origin[:] = [float(x) for x in m.rel_origin]
            marr[i].rel_size[:] = [float(x) for x in m.rel_size]
            marr[i].nsplit[:] = [int(x) for x in m.nsplit]
        barr = (TbBandDesc * max(1, len(bands)))()
        for i, b in enumerate(bands):
            disp = np.ascontiguousarray(b.dispersion_coeffs, dtype=np.float64)
            self._keep.append(disp)
            barr[i].mesh = meshes.index(b.mesh)
            barr[i].charge = b.charge
            barr[i].statistics = b.statistics
            barr[i].dispersion = dptr(disp)
            barr[i].abs_tol = b.absoluteErrorTolerance
            barr[i].rel_tol = b.relativeErrorTolerance
            barr[i].penalisation = b.penalisationUnphysicalPopulation
            barr[i].constrained = 1 if b.constrained else 0
            if b.constrained:
                # a time-dependent population is installed as a callback after
                # creation (tb_set_constraint_fn); the description holds zeros
                cp = (np.zeros(b.mesh.ne * 3) if callable(b.constrainedPopulation)
                      else np.ascontiguousarray(b.constrainedPopulation, dtype=np.float64))
                self._keep.append(cp)
                barr[i].constrained_population = dptr(cp)
            barr[i].drift_velocity[:] = [float(x) for x in b.drift_velocity]
        carr = (TbChannelDesc * max(1, len(channels)))()
        for i, c in enumerate(channels):
            carr[i].nlegs = c.nlegs
            for l in range(c.nlegs):
                carr[i].band[l] = c.legBandNumber[l]
                carr[i].dir[l] = c.legDirection[l]
            carr[i].amplitude = c.amplitude
            carr[i].n_mc = c.numMCPoints
            carr[i].min_det = c.minimumDeterminant
            carr[i].threshold = c.scattElemeThreshold
            umk = np.ascontiguousarray(c.umklappUnitVectors, dtype=np.float64).reshape(-1)
            mc = np.ascontiguousarray(c.mc_points, dtype=np.float64)
            mcp = np.ascontiguousarray(c.mc_points_precalc, dtype=np.float64)
            self._keep += [umk, mc, mcp]
            carr[i].n_umklapp = umk.size // 2
            carr[i].umklapp = dptr(umk)
            carr[i].mc_points = dptr(mc)
            carr[i].mc_points_precalc = dptr(mcp)
            if c.tuples is not None:
                t = np.ascontiguousarray(c.tuples, dtype=np.int32)
                u = np.ascontiguousarray(c.tuple_umklapp, dtype=np.int32)
                self._keep += [t, u]
                carr[i].n_tuples = u.size
                carr[i].tuples = iptr(t)
                carr[i].tuple_umklapp = iptr(u)
            else:
                carr[i].n_tuples = 0
        d.n_meshes = len(meshes)
        d.meshes = C.cast(marr, C.POINTER(TbMeshDesc))
        d.n_bands = len(bands)
        d.bands = C.cast(barr, C.POINTER(TbBandDesc))
        d.n_channels = len(channels)
        d.channels = C.cast(carr, C.POINTER(TbChannelDesc))
        self._keep += [marr, barr, carr]
        self.desc = d

    def ref(self):
        return C.byref(self.desc)
