"""The C-ABI library loads without a GPU and exports every symbol that
include/nb6b200.h declares (no compute calls here)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "nb6b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z][a-z0-9_]*_)\s*\(", text)))


def test_header_declares_reference_abi():
    syms = declared_symbols()
    for s in ("gpunb_open_", "gpunb_close_", "gpunb_send_", "gpunb_regf_", "gpunb_profile_",
              "gpunb_devinit_", "gpupot_", "irr_simd_open_", "irr_simd_close_",
              "irr_simd_set_jp_", "irr_simd_set_list_", "irr_simd_firr_vec_",
              "irr_simd_profile_"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import nb6b200
    lib = nb6b200.load_cdll()          # loads on a CPU-only machine too
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared_symbols()) == set(nb6b200.ABI_SYMBOLS)


def test_exports_are_plain_c_symbols():
    import nb6b200
    out = subprocess.run(["nm", "-D", "--defined-only", nb6b200.library_path()],
                         capture_output=True, text=True, check=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    for s in declared_symbols():
        assert s in exported, s


def test_missing_library_fails_loudly(tmp_path, monkeypatch):
    import nb6b200
    monkeypatch.setattr(nb6b200, "LIB_PATH", str(tmp_path / "nope.so"))
    monkeypatch.setattr(nb6b200, "_LIB", None)
    with pytest.raises(RuntimeError):
        nb6b200.load_cdll()
