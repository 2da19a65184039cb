"""The no-allocation error-norm entry point, checked against the existing one.

tb_band_relative_error_noalloc serves callers that cannot allocate device
memory when they call in (their device memory belongs to their own pool
allocator, or they cannot afford the implicit synchronisation of
cudaMalloc/cudaFree): it keeps its partial sums in a fixed static device array.
Here it is called twice in a row through the C ABI on caller-owned device
buffers and must agree with tb_relative_error (which uses the handle's own
scratch) within the error-norm tolerance of the other parity tests.
"""
import ctypes as C

import numpy as np
import pytest

from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _bind(lib):
    f = lib.tb_band_relative_error_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double,
                  C.c_double, C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("n", [16, 24])
def test_noalloc_error_norm_matches_existing_entry_point(gpu_lib, n):
    import torch
    fn = _bind(gpu_lib)
    mat = W.parabolic_ee(n)
    band = mat.bands[0]
    band.penalisationUnphysicalPopulation = 0.5
    eng = E.Engine(mat)
    rng = np.random.default_rng(n)
    outs = []
    for call in range(2):
        pop = W.initial_status(mat, seed=call).vec
        pop = pop + 0.05 * rng.standard_normal(pop.size)     # some unphysical values
        err = 1e-7 * rng.standard_normal(pop.size)
        ref = eng.relative_error(err, pop)
        e_d = torch.tensor(err, device="cuda")
        p_d = torch.tensor(pop, device="cuda")
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = fn(e_d.data_ptr(), p_d.data_ptr(), band.mesh.ne, band.mesh.elemVolume, band.statistics,
                band.relativeErrorTolerance, band.absoluteErrorTolerance, band.penalisationUnphysicalPopulation,
                out.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == 0, gpu_lib.tb_last_error()
        got = float(out.item())
        assert abs(got - ref) <= 1e-13 * abs(ref), (got, ref)
        outs.append(got)
    assert outs[0] != outs[1]


def test_noalloc_rejects_sizes_beyond_the_limit(gpu_lib):
    fn = _bind(gpu_lib)
    gpu_lib.tb_last_error.restype = C.c_char_p
    rc = fn(C.c_void_p(8), C.c_void_p(8), 1048577, 1.0, -1.0, 1e-3, 1e-3, 0.0, C.c_void_p(8), None)
    assert rc == 9
    assert b"static scratch limit" in gpu_lib.tb_last_error()


def test_noalloc_on_a_side_stream_without_penalisation(gpu_lib):
    """Two calls in a row on a non-default stream, with the penalisation
    term switched off (penalisation 0 skips it in both entry points)."""
    import torch
    fn = _bind(gpu_lib)
    mat = W.parabolic_ee(12)
    band = mat.bands[0]
    band.penalisationUnphysicalPopulation = 0.0
    eng = E.Engine(mat)
    rng = np.random.default_rng(7)
    side = torch.cuda.Stream()
    for call in range(2):
        pop = W.initial_status(mat, seed=10 + call).vec + 0.05 * rng.standard_normal(3 * band.mesh.ne)
        err = 1e-7 * rng.standard_normal(pop.size)
        ref = eng.relative_error(err, pop)
        e_d = torch.tensor(err, device="cuda")
        p_d = torch.tensor(pop, device="cuda")
        out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = fn(e_d.data_ptr(), p_d.data_ptr(), band.mesh.ne, band.mesh.elemVolume, band.statistics,
                band.relativeErrorTolerance, band.absoluteErrorTolerance, 0.0, out.data_ptr(),
                C.c_void_p(side.cuda_stream))
        side.synchronize()
        assert rc == 0, gpu_lib.tb_last_error()
        assert abs(float(out.item()) - ref) <= 1e-13 * abs(ref)
