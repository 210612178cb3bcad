"""The C ABI boundary: the library loads, exports every entry point that
include/emses_gpu.h declares, and the ctypes mirror matches the C layouts.
No compute call is made here (CPU only)."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

from ctca_b200 import emses

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "emses_gpu.h"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(emsesg_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_reference_entry_points():
    names = header_functions()
    for ref_name in ("grdcrt", "psolve1", "psolve2", "charge", "spsort"):
        assert f"emsesg_{ref_name}" in names


def test_library_exports_every_declared_symbol():
    lib = emses.load_library()
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(emses.library_path())], capture_output=True, text=True)
    exported = set(re.findall(r"\bT (emsesg_\w+)", out.stdout))
    assert set(header_functions()) <= exported


def test_python_mirror_covers_the_header():
    assert sorted(emses.declared_symbols()) == header_functions()


def _c_layout():
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "emses_gpu.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(emsesg_particle), sizeof(emsesg_counter), sizeof(emsesg_config),
         sizeof(emsesg_body), sizeof(emsesg_plasma));
  printf("%zu %zu %zu %zu\n", offsetof(emsesg_config, rng_seed), offsetof(emsesg_config, body),
         offsetof(emsesg_config, capacity), offsetof(emsesg_counter, chgacm));
  return 0;
}
'''
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = Path(d) / "l.c"
        c.write_text(src)
        exe = Path(d) / "l"
        subprocess.run(["gcc", "-I", str(ROOT / "include"), "-o", str(exe), str(c)], check=True)
        out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    return [int(x) for x in out]


def test_struct_layouts_match_c():
    sp, sc, scfg, sb, spl, o_seed, o_body, o_cap, o_chg = _c_layout()
    assert sp == 64 == emses.PARTICLE_DTYPE.itemsize
    assert sc == ctypes.sizeof(emses.Counter) == 11240  # Fortran sequence type `counter`
    assert scfg == ctypes.sizeof(emses.Config)
    assert sb == ctypes.sizeof(emses.Body)
    assert spl == ctypes.sizeof(emses.Plasma)
    assert o_seed == emses.Config.rng_seed.offset
    assert o_body == emses.Config.body.offset
    assert o_cap == emses.Config.capacity.offset
    assert o_chg == emses.Counter.chgacm.offset


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setenv("EMSESG_LIB", str(tmp_path / "nope.so"))
    monkeypatch.setattr(emses, "_lib", None)
    with pytest.raises(ImportError):
        emses.load_library()


def test_fx_row_slots_match_the_header():
    import re
    from ctca_b200.emses import FX_ROW_SLOTS
    text = (Path(__file__).resolve().parent.parent / "include" / "emses_gpu.h").read_text()
    assert int(re.search(r"#define EMSESG_FX_ROW_SLOTS (\d+)", text).group(1)) == FX_ROW_SLOTS
