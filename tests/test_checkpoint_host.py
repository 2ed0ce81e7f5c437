"""The checkpoint header's layout as C lays it out (compiled here with gcc
from include/exo_b200.h) and as the Python mirror reads it."""
import ctypes
import os
import subprocess

import pytest

from exocubed_b200 import _native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "exo_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(exo_checkpoint_header), sizeof(exo_config),
         offsetof(exo_checkpoint_header, values), offsetof(exo_checkpoint_header, time),
         offsetof(exo_checkpoint_header, ncycle), offsetof(exo_checkpoint_header, invalid),
         offsetof(exo_checkpoint_header, cfg));
  return 0;
}
"""


def test_header_layout_matches_c(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    r = subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o",
                        str(exe)], capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr)
    got = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                          check=True).stdout.split()]
    H = nat.CheckpointHeader
    want = [ctypes.sizeof(H), ctypes.sizeof(nat.ExoConfig), H.values.offset, H.time.offset,
            H.ncycle.offset, H.invalid.offset, H.cfg.offset]
    assert got == want
    assert got[0] == 512


def test_header_parse():
    h = nat.CheckpointHeader()
    h.magic = b"EXOCKPT1"
    h.version = 1
    h.header_bytes = 512
    h.time, h.dt, h.ncycle = 1.5, 0.25, 7
    h.cfg.N, h.cfg.L, h.cfg.eqn = 8, 12, 1
    d = nat.checkpoint_header(bytes(h) + b"\0" * 64)
    assert d["magic"] == b"EXOCKPT1" and d["ncycle"] == 7 and d["time"] == 1.5
    assert d["cfg"]["N"] == 8 and d["cfg"]["L"] == 12
    with pytest.raises(ValueError):
        nat.checkpoint_header(b"\0" * 100)
