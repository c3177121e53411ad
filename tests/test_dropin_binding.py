"""The reference's own ctypes binding loads this library unchanged (CPU only).

The binding binds ~300 symbols eagerly, most outside the channelizer path,
so the drop-in is a link-only composite: this library first, the reference
library (built from its sources into oracle/_ref) second. The dynamic loader
then resolves the channelizer path from this library and everything else
from the reference.

The reference's source tree (for its binding, python/atkdsp) is named by the
ATKDSP_REFERENCE environment variable; the test is skipped where it is not
set or the binding is absent. No GPU call is made: load(), the ABI check and
symbol binding need none.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

import pytest

from conftest import ROOT

REF_PY = Path(os.environ.get("ATKDSP_REFERENCE", "/nonexistent")) / "python"
REF_SO = ROOT / "oracle" / "_ref" / "libatkdsp_ref.so"
OUR_SO = ROOT / "atkdsp_b200" / "lib" / "libatkdsp_b200.so"

pytestmark = pytest.mark.skipif(not (REF_PY / "atkdsp" / "__init__.py").exists() or not REF_SO.exists(),
                                reason="reference binding or reference library not present")


def test_reference_binding_loads_the_composite(tmp_path):
    gcc = shutil.which("gcc", path="/usr/bin") or "gcc"
    shutil.copy(REF_SO, tmp_path / "libatkdsp_cpu.so")
    composite = tmp_path / "atkdsp.so"
    subprocess.run([gcc, "-shared", "-o", str(composite), "-Wl,--no-as-needed",
                    f"-L{OUR_SO.parent}", f"-L{tmp_path}", "-latkdsp_b200", "-l:libatkdsp_cpu.so",
                    f"-Wl,-rpath,{OUR_SO.parent}", f"-Wl,-rpath,{tmp_path}"], check=True)
    probe = f"""
import sys, ctypes
sys.path.insert(0, {str(REF_PY)!r})
import atkdsp
lib = atkdsp.load()
assert lib.atkdsp_abi_version() == 26
info = atkdsp.build_info()
assert "abi 26" in info and "b200" in info, info
ours = ctypes.CDLL({str(OUR_SO)!r})
for name in ("atkdsp_pfb_create", "atkdsp_pfb_process_n", "atkdsp_unpack_dc",
             "atkdsp_pfb_cov_accumulate", "atkdsp_pfb_channel_power", "atkdsp_osx_process_n",
             "atkdsp_cfar_create", "atkdsp_cfar_process", "atkdsp_cfar_alpha"):
    a = ctypes.cast(getattr(lib, name), ctypes.c_void_p).value
    b = ctypes.cast(getattr(ours, name), ctypes.c_void_p).value
    assert a == b, name
assert lib.atkdsp_nco_mix is not None            # outside the path: the reference's
a, et = atkdsp.cfar_alpha("ca", 16, 1e-6)        # the binding's solver call, answered by this library
assert abs(a - 17.27764883379317) < 1e-12, a
print("ok", info)
"""
    env = dict(os.environ, ATKDSP_LIB=str(composite))
    r = subprocess.run([sys.executable, "-c", probe], env=env, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.startswith("ok")
