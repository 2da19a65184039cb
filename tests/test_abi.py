"""C ABI: the library loads, exports every function include/*.h declares,
and the ctypes mirror has the C struct layout.  No device calls."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

from tortoise_b200 import abi
from tortoise_b200 import engine

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(tb_[a-z_0-9]+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = engine.lib()
    names = declared_functions()
    assert "tb_create" in names and "tb_dp45_integrate" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "tortoise_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(tb_region), sizeof(tb_mesh_desc), sizeof(tb_band_desc),
         sizeof(tb_channel_desc), sizeof(tb_problem_desc));
  printf("%zu %zu %zu\n", offsetof(tb_channel_desc, umklapp), offsetof(tb_channel_desc, n_tuples),
         offsetof(tb_band_desc, drift_velocity));
  printf("%zu %zu %zu %zu\n", sizeof(tb_options), sizeof(tb_dp45_stats), sizeof(tb_adjoint_stats),
         offsetof(tb_adjoint_stats, status));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split()
    got = [int(x) for x in out]
    want = [C.sizeof(abi.TbRegion), C.sizeof(abi.TbMeshDesc), C.sizeof(abi.TbBandDesc),
            C.sizeof(abi.TbChannelDesc), C.sizeof(abi.TbProblemDesc),
            abi.TbChannelDesc.umklapp.offset, abi.TbChannelDesc.n_tuples.offset,
            abi.TbBandDesc.drift_velocity.offset, C.sizeof(engine.Options), C.sizeof(engine.DP45Stats),
            C.sizeof(engine.AdjointStats), engine.AdjointStats.status.offset]
    assert got == want


def test_create_without_device_fails_cleanly():
    """With no CUDA device tb_create must fail with TB_ERR_NO_DEVICE, never
    fall back to the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("device present")
    from tortoise_b200 import workloads as W
    mat = W.parabolic_ee(3)
    with pytest.raises(engine.TortoiseError) as ei:
        engine.Engine(mat)
    assert ei.value.rc == 7


def test_shard_ranges_partition_the_tuple_list():
    """tb_shard_range (host arithmetic): for every rank count the parts are
    contiguous, cover [0, n), start on 128-tuple boundaries and differ by at
    most one tile; bad arguments are refused."""
    from tortoise_b200 import engine as E
    for n in (0, 5, 128, 1000, 12345, 9_800_000, 2**40 + 77):
        for R in (1, 2, 3, 4, 7, 8):
            parts = [E.shard_range(n, r, R) for r in range(R)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            for (b, e), (b2, _) in zip(parts, parts[1:]):
                assert e == b2 and b <= e
            for b, _ in parts:
                assert b % 128 == 0 or b == n
            sizes = [e - b for b, e in parts]
            assert max(sizes) - min(sizes) <= 128 + (n % 128 if n < 128 * R else 0)
    for args in ((10, 2, 2), (10, -1, 2), (10, 0, 0), (-1, 0, 1)):
        with pytest.raises(E.TortoiseError):
            E.shard_range(*args)
