"""A plain C program as the host of the library (what a TORTOISE shim is):
tests/c_host_rhs.c builds the problem description from raw arrays and calls
tb_create / tb_rhs / tb_dp45_integrate with host pointers.  Its right-hand
side and its integration must equal the Python binding's: the same library,
so the only differences are the summation order of FP64 atomics, 1e-13 on
the right-hand side and, amplified by the step controller as in the parity
tests, 1e-11 on the dense outputs and 1e-9 on the final state."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _write_input(path, mat, f0, t_final, dense_step, max_dense):
    m = mat.meshes[0]
    g = mat.region.gvec
    with open(path, "wb") as fh:
        fh.write(struct.pack("<6d", *mat.region.origin, g[0, 0], g[1, 0], g[0, 1], g[1, 1]))
        fh.write(struct.pack("<4d", *m.rel_origin, *m.rel_size) + struct.pack("<2i", *m.nsplit))
        fh.write(struct.pack("<i", len(mat.bands)))
        for b in mat.bands:
            assert b.mesh is m and not b.constrained
            fh.write(struct.pack("<6d", b.charge, b.statistics, b.absoluteErrorTolerance, b.relativeErrorTolerance,
                                 *b.drift_velocity))
            fh.write(struct.pack("<i", b.mesh.ne))
            fh.write(np.ascontiguousarray(b.dispersion_coeffs, dtype="<f8").tobytes())
        fh.write(struct.pack("<i", len(mat.channels)))
        for c in mat.channels:
            L = c.nlegs
            fh.write(struct.pack("<i", L) + struct.pack("<%di" % L, *c.legBandNumber)
                     + struct.pack("<%di" % L, *c.legDirection))
            fh.write(struct.pack("<d", c.amplitude) + struct.pack("<i", c.numMCPoints))
            fh.write(struct.pack("<2d", c.minimumDeterminant, c.scattElemeThreshold))
            umk = np.ascontiguousarray(c.umklappUnitVectors, dtype="<f8").reshape(-1)
            fh.write(struct.pack("<i", umk.size // 2) + umk.tobytes())
            fh.write(np.ascontiguousarray(c.mc_points, dtype="<f8").tobytes())
            fh.write(np.ascontiguousarray(c.mc_points_precalc, dtype="<f8").tobytes())
        fh.write(struct.pack("<q", f0.size) + np.ascontiguousarray(f0, dtype="<f8").tobytes())
        fh.write(struct.pack("<2d", t_final, dense_step) + struct.pack("<q", max_dense))


def test_c_host_matches_the_python_binding(gpu_lib, tmp_path):
    exe = tmp_path / "c_host_rhs"
    subprocess.check_call(["gcc", "-O2", "-std=c99", "-I" + os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c_host_rhs.c"), "-o", str(exe),
                           "-L" + os.path.dirname(E.LIB_PATH), "-ltortoise_b200",
                           "-Wl,-rpath," + os.path.dirname(E.LIB_PATH)])
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=True, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    f0 = W.initial_status(mat, kT=0.1, seed=8).vec
    t_final, dense_step, max_dense = 0.2, 0.1, 4
    _write_input(tmp_path / "in.bin", mat, f0, t_final, dense_step, max_dense)
    subprocess.check_call([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")])
    raw = np.fromfile(tmp_path / "out.bin", dtype="<f8")
    n = f0.size
    rhs = raw[:n]
    stats = np.frombuffer(raw[n:n + 4].tobytes(), dtype="<i8")
    dense = raw[n + 4:n + 4 + max_dense * n].reshape(max_dense, n)
    y = raw[n + 4 + max_dense * n:]
    eng = E.Engine(mat)
    assert rel_l2(rhs, eng.rhs(f0)) < 1e-13
    ref = eng.dp45(f0, 0.0, t_final, dense_step, max_dense=max_dense)
    assert [int(x) for x in stats] == [ref["attempts"], ref["accepted"], ref["rejected"], ref["n_dense"]]
    nd = int(stats[3])
    assert rel_l2(dense[:nd], ref["dense"]) < 1e-11
    assert rel_l2(y, ref["y"]) < 1e-9
