"""The Gauss quadrature constants against the reference's own header.

oracle/_ref/libref_gauss.so reads the order-2 rules out of the reference's
include/Geometry/GeometryCore/GaussQuadratureConst.hpp, compiled where it lies
by `make -C oracle ref`.  The mass matrix, the error norm and the drift's
surface terms all integrate with these 14-digit constants (not exact thirds),
so the oracle's tables (oracle/tortoise_oracle.cpp) and the CUDA library's
(TB_GP2_*, TB_GW2, TB_GP1_* in tortoise_b200/csrc/tb_common.cuh) must hold the
same doubles.  Skipped where the reference tree was not there to build from.
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT

REF = os.path.join(ROOT, "oracle", "_ref", "libref_gauss.so")
pytestmark = pytest.mark.skipif(not os.path.exists(REF), reason="oracle/_ref not built (no reference tree)")
DP = C.POINTER(C.c_double)


def _reference():
    L = C.CDLL(REF)
    L.ref_gauss_triangle_order2.argtypes = [DP, DP]
    L.ref_gauss_interval_order2.argtypes = [DP, DP]
    tp, tw, ip, iw = np.zeros(6), np.zeros(3), np.zeros(2), np.zeros(2)
    L.ref_gauss_triangle_order2(tp.ctypes.data_as(DP), tw.ctypes.data_as(DP))
    L.ref_gauss_interval_order2(ip.ctypes.data_as(DP), iw.ctypes.data_as(DP))
    return tp.reshape(3, 2), tw, ip, iw


def test_oracle_gauss_rules_are_the_reference_constants():
    tp, tw, ip, _ = _reference()
    op, ow, oi = np.zeros(6), np.zeros(3), np.zeros(2)
    oracle.lib().or_gauss_constants(op.ctypes.data_as(DP), ow.ctypes.data_as(DP), oi.ctypes.data_as(DP))
    assert np.array_equal(op.reshape(3, 2), tp)
    assert np.array_equal(ow, tw)
    assert np.array_equal(oi, ip)
    # the 14-digit values, not exact thirds
    assert tw[0] == 0.33333333333333 and tw[0] != 1.0 / 3.0


def test_device_gauss_rules_are_the_reference_constants():
    tp, tw, ip, _ = _reference()
    src = open(os.path.join(ROOT, "tortoise_b200", "csrc", "tb_common.cuh")).read()
    macro = {m.group(1): float(m.group(2)) for m in re.finditer(r"#define (TB_G\w+) ([0-9.eE+-]+)", src)}
    # the triangle rule's nodes are (A, A), (B, A), (A, B)
    a, b = macro["TB_GP2_A"], macro["TB_GP2_B"]
    assert np.array_equal(np.array([[a, a], [b, a], [a, b]]), tp)
    assert np.array_equal(np.full(3, macro["TB_GW2"]), tw)
    assert np.array_equal(np.array([macro["TB_GP1_0"], macro["TB_GP1_1"]]), ip)
