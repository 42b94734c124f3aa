"""The reference's C ABI acceptance test (capi/test/roundtrip.c), compiled
unmodified against include/quoin.h and libquoin_b200.so by `make -C oracle ref`
(the binary travels with the built library; skipped where it was not built)."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "capi_roundtrip")


@pytest.mark.gpu
def test_reference_capi_roundtrip_passes():
    if not os.path.exists(BIN):
        pytest.skip("oracle/_ref/capi_roundtrip not built (needs the reference tree at build time)")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "All C ABI tests passed." in r.stdout
