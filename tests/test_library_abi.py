"""The drop-in boundary, checked without a GPU (CPU only).

The in-tree library must load on any host, report the reference's ABI (26)
and export every entry point that include/*.h declares -- and nothing the
headers do not declare. Compute needs a GPU: on a host without one, create
returns NULL and the binding raises, rather than falling back to the CPU.
"""

from __future__ import annotations

import re
import subprocess

import pytest

import atkdsp_b200 as ak
from conftest import ROOT

HEADERS = sorted((ROOT / "include").glob("*.h"))


def _declared() -> set:
    names = set()
    for h in HEADERS:
        text = h.read_text()
        for m in re.finditer(r"ATKDSP_API\s+[^;(]*?\b(atkdsp_\w+)\s*\(", text, re.S):
            names.add(m.group(1))
    return names


def _exported() -> set:
    out = subprocess.run(["nm", "-D", "--defined-only", str(ak.LIB_FILE)], check=True,
                         capture_output=True, text=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_headers_declare_the_reference_surface():
    d = _declared()
    for name in ("atkdsp_abi_version", "atkdsp_version_string", "atkdsp_build_info",
                 "atkdsp_bytes_per_sample", "atkdsp_set_threads", "atkdsp_get_threads",
                 "atkdsp_unpack", "atkdsp_unpack_dc", "atkdsp_pfb_create", "atkdsp_pfb_destroy",
                 "atkdsp_pfb_reset", "atkdsp_pfb_nchan", "atkdsp_pfb_out_rate",
                 "atkdsp_pfb_out_hops", "atkdsp_pfb_process", "atkdsp_pfb_process_n",
                 "atkdsp_pfb_block_origin", "atkdsp_pfb_group_delay", "atkdsp_pfb_set_cal",
                 "atkdsp_pfb_describe", "atkdsp_pfb_cov_accumulate", "atkdsp_pfb_cov_reset",
                 "atkdsp_pfb_channel_power", "atkdsp_osx_create", "atkdsp_osx_destroy",
                 "atkdsp_osx_reset", "atkdsp_osx_add", "atkdsp_osx_retune", "atkdsp_osx_remove",
                 "atkdsp_osx_channels", "atkdsp_osx_chan_rate", "atkdsp_osx_out_max",
                 "atkdsp_osx_process", "atkdsp_osx_process_n", "atkdsp_osx_describe"):
        assert name in d, name


def test_library_exports_exactly_the_declared_symbols():
    d, e = _declared(), _exported()
    assert d - e == set(), f"declared but not exported: {sorted(d - e)}"
    assert e - d == set(), f"exported but not declared: {sorted(e - d)}"


def test_library_loads_and_reports_abi_26():
    lib = ak.load()
    assert lib.atkdsp_abi_version() == 26
    assert ak.version() == "0.25.1"
    assert "abi 26" in ak.build_info()


def test_identity_helpers():
    for f, n in (("cu8", 2), ("ci8", 2), ("ci16", 4), ("ci16q11", 4), ("cf32", 8)):
        assert ak.bytes_per_sample(f) == n
    assert ak.load().atkdsp_bytes_per_sample(99) == 0
    before = ak.get_threads()
    assert ak.set_threads(3) == 3 and ak.get_threads() == 3
    ak.set_threads(0)
    assert ak.get_threads() == before


def test_create_rejects_bad_arguments_before_touching_a_device():
    lib = ak.load()
    for args in ((0.0, 64, 2, 12, 80.0, 1), (1e6, 1, 1, 12, 80.0, 1), (1e6, 64, 3, 12, 80.0, 1),
                 (1e6, 64, 2, 1, 80.0, 1), (1e6, 64, 2, 12, 80.0, 0), (1e6, 8192, 2, 12, 80.0, 1)):
        assert not lib.atkdsp_pfb_create(*args), args
    for args in ((0.0, 4096, 80.0, 1), (1e6, 32, 80.0, 1), (1e6, 100, 80.0, 1), (1e6, 4096, 80.0, 0),
                 (1e6, 1 << 25, 80.0, 1)):
        assert not lib.atkdsp_osx_create(*args), args
    # void / query calls ignore a NULL handle like the reference's
    lib.atkdsp_osx_destroy(None)
    lib.atkdsp_osx_reset(None)
    assert lib.atkdsp_osx_channels(None) == 0 and lib.atkdsp_osx_chan_rate(None, 0) == 0.0
    assert lib.atkdsp_osx_out_max(None, 0, 100) == 0
    assert lib.atkdsp_osx_add(None, 0.0, 1.0, 1.0) == -1 and lib.atkdsp_osx_remove(None, 0) == -1


def test_no_cpu_fallback_without_a_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(ak.AtkDspError):
        ak.Pfb(2.4e6, 64, 2, 12)
    with pytest.raises(ak.AtkDspError):
        ak.unpack(b"\x00\x01\x02\x03", "ci16")
    with pytest.raises(ak.AtkDspError):
        ak.Osx(2.4e6, 4096)
