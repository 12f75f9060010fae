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


def write_codewords(path, seed=8):
    """Transport blocks for the pusch_decoder check: per TB its parameters and two transmissions
    (rv 0 as new data, then rv 2 soft-combined), soft bits of the project's transmit-side UL-SCH
    codec (codec.ulsch_encode) through a noisy BPSK-like channel, quantised to the LLR range.
    The noise is chosen so that some first transmissions fail and combining rescues them."""
    import struct

    import numpy as np

    from pusch_b200 import codec
    rng = np.random.default_rng(seed)
    # (TBS, base graph, Qm, layers, channel symbols): a 20 MHz QPSK TB, a small CRC16 TB, a
    # multi-codeblock 64QAM TB and the 100 MHz 256QAM 2-layer TB (50 codeblocks).
    cases = [(5888, 1, 2, 1, 13 * 612), (1320, 2, 4, 1, 12 * 72), (40976, 1, 6, 2, 2 * 12 * 600),
             (417976, 1, 8, 2, 2 * 12 * 3276), (3824, 2, 2, 1, 12 * 204), (24576, 1, 4, 2, 2 * 12 * 700)]
    out = [struct.pack("<i", len(cases))]
    for t, (tbs, bg, qm, nl, ncs) in enumerate(cases):
        seg = codec.segment_tx(tbs, bg, qm, nl, ncs)
        tb = rng.integers(0, 2, tbs, dtype=np.uint8)
        g = ncs * qm
        out.append(struct.pack("<8i", tbs // 8, bg, qm, nl, 0, g, seg["nof_cbs"], 2))
        sigma = [0.95, 0.7, 0.85, 0.75, 1.1, 0.8][t]
        for rv, nd in ((0, 1), (2, 0)):
            cw = codec.ulsch_encode(tb, bg, qm, nl, ncs, seg, rv=rv)
            y = (1.0 - 2.0 * cw) + sigma * rng.standard_normal(g)
            llr = np.clip(np.rint(y * 2 / sigma ** 2 * 2.5), -120, 120).astype(np.int8)
            out.append(struct.pack("<2i", rv, nd))
            out.append(llr.tobytes())
    with open(path, "wb") as f:
        f.write(b"".join(out))


@needs_check
@pytest.mark.gpu
def test_adapters_match_reference_implementations(tmp_path):
    cw = os.path.join(str(tmp_path), "codewords.bin")
    write_codewords(cw)
    r = subprocess.run([CHECK, cw], capture_output=True, text=True, timeout=900)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    for iface in ("ldpc_decoder", "ldpc_rate_dematcher", "crc_calculator", "demodulation_mapper", "channel_equalizer",
                  "port_channel_estimator", "pusch_decoder", "resident_decoder"):
        assert any(line.startswith(iface) and " OK " in line for line in r.stdout.splitlines()), iface


DAPP_CHECK = os.path.join(ROOT, "oracle", "_ref", "dapp_check")
DAPP_MODULE = os.path.join(ROOT, "ocudu-dapp-platform_b200", "adapters", "_lib", "libpg_dapp_b200.so")
needs_dapp = pytest.mark.skipif(not (os.path.exists(DAPP_CHECK) and os.path.exists(DAPP_MODULE)),
                                reason="oracle/_ref/dapp_check or the dApp module not built")


@needs_dapp
def test_dapp_module_descriptor_passes_reference_validator():
    """The dApp plug-in module loads through ocudu_dapp_query_v1 and the reference's own ABI
    validator accepts its descriptor: two Class-A interfaces (channel estimator v1, receiver v1)."""
    r = subprocess.run([DAPP_CHECK, DAPP_MODULE, "--describe"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert any(line.startswith("dapp_module") and " OK " in line for line in r.stdout.splitlines())


@needs_dapp
@pytest.mark.gpu
def test_dapp_module_matches_reference_chain():
    """The module's channel estimator and receiver, invoked with the host hooks' tensors, against the
    reference's native port_channel_estimator / channel_equalizer / demodulation_mapper."""
    r = subprocess.run([DAPP_CHECK, DAPP_MODULE], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    for name in ("dapp_module", "dapp_channel_estimator", "dapp_receiver", "dapp_bypass", "dapp_lifecycle"):
        assert any(line.startswith(name) and " OK " in line for line in r.stdout.splitlines()), name
