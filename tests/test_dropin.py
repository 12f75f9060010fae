"""Drop-in check of the C++ adapters (ocudu-dapp-platform_b200/adapters): the reference's own PHY
interfaces served by the reference's compiled code and by the adapters over the GPU library, on the
same seeded inputs (tests/dropin/adapter_check.cpp, built into oracle/_ref by oracle/Makefile)."""
import os
import subprocess

import pytest

from conftest import ROOT, has_gpu

CHECK = os.path.join(ROOT, "oracle", "_ref", "adapter_check")

needs_check = pytest.mark.skipif(not os.path.exists(CHECK), reason="oracle/_ref/adapter_check not built")


@needs_check
@pytest.mark.skipif(has_gpu(), reason="checks the behaviour without a GPU")
def test_adapters_fail_loudly_without_gpu():
    """No CPU fallback behind the adapters: without a device the first adapter ends the process."""
    r = subprocess.run([CHECK], capture_output=True, text=True, timeout=120)
    assert r.returncode != 0
    assert "pusch_b200: pg_create" in (r.stdout + r.stderr)


@needs_check
@pytest.mark.gpu
def test_adapters_match_reference_implementations():
    r = subprocess.run([CHECK], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    for iface in ("ldpc_decoder", "ldpc_rate_dematcher", "crc_calculator", "demodulation_mapper", "channel_equalizer"):
        assert any(line.startswith(iface) and " OK " in line for line in r.stdout.splitlines()), iface
