"""The bounded device wait of the moment-tensor contractions.

Every thread block of k_collision_tensor / k_collision_runs waits for its
staged tiles of moments with a poll limit (tb_set_copy_wait_limit).  With the
limit at 0 every wait gives up at once: the block records the failure in the
handle's flag, waits -- with its own, unchanged bound -- for the copies it has
in flight, and leaves its tiles out.  Nothing faults or hangs.  The
synchronising calls then report TB_ERR_TIMEOUT, and with the limit restored the
same handle gives its normal results again."""
import numpy as np
import pytest

from conftest import rel_l2
from tortoise_b200 import engine as E
from tortoise_b200 import workloads as W

pytestmark = pytest.mark.gpu
TIMEOUT = 6
DEFAULT_POLLS = 1 << 22


def _eph():
    mat = W.build_material(4, ("P", "D"), (0.2,), ee=False, eph=True, field=(0.1, 0.0), rtol=1e-6, atol=1e-9)
    return mat, W.initial_status(mat, seed=4).vec


@pytest.mark.parametrize("layout", [E.LAYOUT_T64, E.LAYOUT_T40])
def test_single_run_wait_runs_out_and_the_handle_recovers(gpu_lib, layout):
    mat, f0 = _eph()
    e = E.Engine(mat, layout=layout, deterministic=True)
    try:
        ref = e.rhs(f0)
        ref_rates = e.scattering_rates(f0)
        ref_dp = e.dp45(f0, 0.0, 0.1, 0.05)
        e.set_copy_wait_limit(0)
        with pytest.raises(E.TortoiseError) as ex:
            e.rhs(f0)
        assert ex.value.rc == TIMEOUT
        with pytest.raises(E.TortoiseError) as ex:
            e.scattering_rates(f0)
        assert ex.value.rc == TIMEOUT
        r = e.dp45(f0, 0.0, 0.1, 0.05)
        assert r["rc"] == TIMEOUT and r["status"] == TIMEOUT and r["done"] == 1
        e.set_copy_wait_limit(DEFAULT_POLLS)
        assert np.array_equal(e.rhs(f0), ref)
        assert np.array_equal(e.scattering_rates(f0), ref_rates)
        r = e.dp45(f0, 0.0, 0.1, 0.05)
        assert r["rc"] == 0 and r["attempts"] == ref_dp["attempts"]
        assert np.array_equal(r["y"], ref_dp["y"])
    finally:
        e.close()


def test_run_minor_wait_runs_out_and_the_batch_recovers(gpu_lib):
    mats, states = W.ensemble_runs(16, seed=9, Ns=(4,))
    be = E.BatchEngine(mats, layout=E.LAYOUT_T40)
    try:
        for ch in range(len(mats[0].channels)):
            be.set_schedule(ch, 2, runs=8)
        f = np.concatenate(states)
        ref = be.rhs(f)
        be.set_copy_wait_limit(0)
        with pytest.raises(E.TortoiseError) as ex:
            be.rhs(f)
        assert ex.value.rc == TIMEOUT
        be.set_copy_wait_limit(DEFAULT_POLLS)
        assert rel_l2(be.rhs(f), ref) < 1e-13
    finally:
        be.close()


def test_wait_limit_is_validated(gpu_lib):
    mat, _ = _eph()
    e = E.Engine(mat, layout=E.LAYOUT_T64)
    try:
        for bad in (-1, 1 << 31):
            with pytest.raises(E.TortoiseError) as ex:
                e.set_copy_wait_limit(bad)
            assert ex.value.rc == 8
    finally:
        e.close()
