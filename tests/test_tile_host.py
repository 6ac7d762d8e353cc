"""CPU check of the banded kernel's warp-tile code (band_tile.cuh): the
kernel's loop emulated lane by lane on the host, under AddressSanitizer,
with every buffer exactly sized and misaligned on purpose; outputs compared
with the oracle.  This is how the kernel's indexing is checked before it
runs on a GPU."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
SRC = ROOT / "tests" / "harness" / "tile_host.cpp"
SO = ROOT / "tests" / "_build" / "libtile_host_asan.so"


def test_tile_emulation_under_asan():
    SO.parent.mkdir(exist_ok=True)
    deps = [SRC, ROOT / "saruman_b200" / "csrc" / "band_tile.cuh",
            ROOT / "saruman_b200" / "csrc" / "saru_core.cuh"]
    if not SO.exists() or SO.stat().st_mtime < max(d.stat().st_mtime for d in deps):
        subprocess.run(["g++", "-O1", "-g", "-std=c++17", "-shared", "-fPIC",
                        "-fsanitize=address", "-fno-omit-frame-pointer", "-o", str(SO),
                        str(SRC)], check=True)
    asan = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True,
                          text=True).stdout.strip()
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0")
    r = subprocess.run([sys.executable, str(ROOT / "tests" / "tile_asan_driver.py"), str(SO)],
                       capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
    assert "BAD 0" in r.stdout


FLANK_CHECK = r'''
#include <stdio.h>
#include "saru_core.cuh"
int main() {
  for (int k = 0; k <= 15; ++k)
    for (int dir = -300; dir <= 300; ++dir) {
      int so, eo, wso = 0, weo = 0;  // the flag meanings of src/hash.c:938-979
      switch (dir) {
        case 1: case 5: weo = k; break;
        case 2: case 6: wso = k; break;
        case 3: case 7: wso = k; weo = k; break;
        default: break;
      }
      saru::flank_of(dir, k, so, eo);
      if (so != wso || eo != weo) { printf("dir %d k %d\n", dir, k); return 1; }
    }
  return 0;
}
'''


def test_flank_of_matches_the_flag_table(tmp_path):
    """The branch-free flank_of gives each flag's start/end gaps exactly as
    the reference's flag table does, for every flag value."""
    src = tmp_path / "flank.cpp"
    src.write_text(FLANK_CHECK)
    exe = tmp_path / "flank"
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", str(ROOT / "saruman_b200" / "csrc"),
                    str(src), "-o", str(exe)], check=True)
    assert subprocess.run([str(exe)]).returncode == 0
