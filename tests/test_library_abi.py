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
                 "atkdsp_osx_process", "atkdsp_osx_process_n", "atkdsp_osx_describe",
                 "atkdsp_cfar_defaults", "atkdsp_cfar_alpha", "atkdsp_cfar_n_eff",
                 "atkdsp_cfar_window_rho2", "atkdsp_cfar_create", "atkdsp_cfar_destroy",
                 "atkdsp_cfar_reset", "atkdsp_cfar_set_mask", "atkdsp_cfar_events_max",
                 "atkdsp_cfar_process", "atkdsp_cfar_flush", "atkdsp_cfar_last", "atkdsp_cfar_info",
                 "atkdsp_cfar_describe", "atkdsp_cfar_stats"):
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
                 (1e6, 64, 2, 1, 80.0, 1), (1e6, 64, 2, 12, 80.0, 0)):
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


def test_cfar_layouts_and_argument_rules_without_a_device():
    """The three CFAR structs have the reference's compiled sizes (96, 64, 88
    bytes: gcc on the reference header gives 96 for the config, whose comment
    says 104); every configuration
    outside the reference's ranges is refused before any device work; the
    NULL-handle rules are the reference's (src/cfar.c:324-340, :745-819)."""
    import ctypes as C
    assert C.sizeof(ak._CfarConfig) == 96 and C.sizeof(ak._CfarEvent) == 64
    assert C.sizeof(ak._CfarCounters) == 88
    lib = ak.load()
    base = ak.cfar_defaults()
    assert base["n_ref"] == 16 and base["n_guard"] == 4 and base["pfa"] == 1e-6 and base["max_tracks"] == 256
    bad = [dict(mode=4), dict(n_ref=0), dict(n_ref=257), dict(n_guard=-1), dict(k_frames=0), dict(k_frames=65),
           dict(looks=0.2), dict(looks=2e4), dict(pfa=0.6), dict(pfa=1e-16), dict(mode=1, os_k=33),
           dict(open_m=4, open_n=3), dict(open_n=65), dict(close_k=0), dict(close_k=1001), dict(merge_gap=-1),
           dict(min_bins=0), dict(max_tracks=0), dict(max_tracks=65537), dict(rho2=(1.0, 0, 0, 0)),
           dict(rho2=(-0.1, 0, 0, 0))]
    for b in bad:
        k = ak._CfarConfig()
        lib.atkdsp_cfar_defaults(C.byref(k))
        for key, v in b.items():
            if key == "rho2":
                k.rho2 = (C.c_double * 4)(*v)
            else:
                setattr(k, key, v)
        assert not lib.atkdsp_cfar_create(1024, C.byref(k)), b
    k = ak._CfarConfig()
    lib.atkdsp_cfar_defaults(C.byref(k))
    for nb in (0, 40, (1 << 24) + 1):
        assert not lib.atkdsp_cfar_create(nb, C.byref(k)), nb
    assert not lib.atkdsp_cfar_create(1024, None)
    lib.atkdsp_cfar_destroy(None)
    lib.atkdsp_cfar_reset(None)
    assert lib.atkdsp_cfar_events_max(None, 10) == 0
    assert lib.atkdsp_cfar_set_mask(None, None) == -1
    assert lib.atkdsp_cfar_flush(None, None, 0) == -1 and lib.atkdsp_cfar_last(None, None, None, None) == -1
    assert lib.atkdsp_cfar_stats(None, None) == -1 and lib.atkdsp_cfar_describe(None, None, 0) == -1
    assert lib.atkdsp_cfar_process(None, None, 0, 0.0, 0.0, None, 0) == -1
    with pytest.raises(ak.AtkDspError):
        ak.cfar_alpha("ca", 0, 1e-6)
    with pytest.raises(ak.AtkDspError):
        ak.cfar_window_rho2([0.0, 0.0, 0.0])


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
    with pytest.raises(ak.AtkDspError):
        ak.Cfar(1024)
