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
