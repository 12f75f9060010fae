"""Seeded synthetic workloads (the project's own simulator; inputs only, never the measured path).

``ldpc_batch``: the LDPC decoder batch workload - codeblocks of random bits with CRC24B attached,
LDPC-encoded (this project's encoder, pusch_b200.codec), BPSK over AWGN at an Eb/N0 drawn per
codeblock, and LLRs 2y/sigma^2 scaled by ``llr_scale`` (LLR units per LSB = 1/llr_scale),
rounded and saturated to int8 +-127. The code rate used for Eb/N0 is R = K/N (CRC included).
"""
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import codec
from .ldpc import BG1, BG2, CodeblockJob, LdpcDecoderConfiguration, bg_k, bg_n_short
from ._native import PG_CRC24B


@dataclass
class LdpcBatch:
    jobs: List[CodeblockJob]
    truth: List[np.ndarray]          # K_b*Z transmitted message bits per codeblock (unpacked)
    ebn0_db: np.ndarray
    base_graphs: np.ndarray
    info_bits: np.ndarray            # information bits per codeblock (K - F - 24)
    params: dict = field(default_factory=dict)


def ldpc_batch(seed=0, n=512, z=384, ebn0_range=(1.0, 3.0), llr_scale=4.0, max_iterations=10, bg_mix=0.5,
               bgs=None):
    """Codeblocks of BG1 (E = N = 66Z, rate 1/3) or BG2 (E = N = 50Z, rate 1/5) mixed by seed."""
    rng = np.random.default_rng(seed)
    if bgs is None:
        bgs = np.where(rng.random(n) < bg_mix, BG1, BG2).astype(np.int32)
    ebn0 = rng.uniform(ebn0_range[0], ebn0_range[1], n)
    jobs, truth = [None] * n, [None] * n
    info = np.zeros(n, np.int64)
    for bg in (BG1, BG2):
        idx = np.nonzero(bgs == bg)[0]
        if idx.size == 0:
            continue
        k = bg_k(bg) * z
        nn = bg_n_short(bg) * z
        msg = codec.attach_crc(PG_CRC24B, rng.integers(0, 2, (idx.size, k - 24), dtype=np.uint8))
        cw = codec.ldpc_encode(bg, z, msg)
        rate = k / nn
        sigma = np.sqrt(1.0 / (2.0 * rate * 10.0 ** (ebn0[idx] / 10.0)))
        y = (1.0 - 2.0 * cw.astype(np.float32)) + sigma[:, None].astype(np.float32) * rng.standard_normal(
            cw.shape, dtype=np.float32)
        llr = np.clip(np.rint(2.0 * y / (sigma[:, None] ** 2) * llr_scale), -127, 127).astype(np.int8)
        cfg = LdpcDecoderConfiguration(base_graph=bg, lifting_size=z, nof_filler_bits=0, nof_crc_bits=24,
                                       max_iterations=max_iterations)
        for t, i in enumerate(idx):
            jobs[i] = CodeblockJob(llr[t], cfg, PG_CRC24B)
            truth[i] = msg[t]
            info[i] = k - 24
    return LdpcBatch(jobs, truth, ebn0, bgs, info,
                     dict(seed=seed, n=n, z=z, ebn0_range=ebn0_range, llr_scale=llr_scale,
                          max_iterations=max_iterations))
