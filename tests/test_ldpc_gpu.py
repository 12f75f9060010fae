"""GPU LDPC decoder parity: bit-exact decoded bits, CRC verdicts and iteration counts against the
reference's outputs (golden fixtures) and the CPU restatement (oracle/pusch_oracle.c)."""
import ctypes

import numpy as np
import pytest

import golden_io
from pusch_b200 import _native, codec, sim
from pusch_b200.ldpc import (CodeblockJob, CrcCalculator, LdpcDecoder, LdpcDecoderConfiguration, make_descriptors,
                             output_bytes)

pytestmark = pytest.mark.gpu


def unpack(b, n):
    return np.unpackbits(np.asarray(b, np.uint8))[:n]


def job_for(c):
    cfg = LdpcDecoderConfiguration(base_graph=c["bg"], lifting_size=c["z"], nof_filler_bits=c["filler"],
                                   nof_crc_bits=16 if c["poly"] == 0 else 24, max_iterations=c["max_iter"])
    return CodeblockJob(c["llrs"], cfg, c["poly"])


def test_golden_batch_bit_exact(batch_decoder):
    cases = golden_io.ldpc_cases()
    outs, iters = batch_decoder.decode_batch([job_for(c) for c in cases])
    for c, o, it in zip(cases, outs, iters):
        k = golden_io.kbits(c["bg"], c["z"])
        assert it == c["iterations"], (c["bg"], c["z"], c["poly"])
        assert (unpack(o, k) == unpack(c["bits"], k)).all(), (c["bg"], c["z"])


def random_jobs(seed, n):
    rng = np.random.default_rng(seed)
    jobs = []
    zs = [8, 13, 16, 26, 36, 64, 72, 104, 120, 176, 192, 208, 224, 240, 256, 288, 320, 352, 384]
    for t in range(n):
        bg = int(rng.integers(1, 3))
        z = int(rng.choice(zs))
        k = golden_io.kbits(bg, z)
        nn = (66 if bg == 1 else 50) * z
        poly = int(rng.choice([0, 1, 2, 2, 255]))
        cpoly = 2 if poly == 255 else poly
        order = 16 if cpoly == 0 else 24
        f = int(rng.integers(0, max(1, min(k - 2 * z - order - 1, k // 4))))
        msg = np.concatenate([codec.attach_crc(cpoly, rng.integers(0, 2, k - f - order, dtype=np.uint8)),
                              np.zeros(f, np.uint8)])
        cw = codec.ldpc_encode(bg, z, msg)
        e = int(rng.integers(k + 2 * z, nn + 1))
        sigma = np.sqrt(1 / (2 * (k / e) * 10 ** (rng.uniform(-1, 4) / 10)))
        llr = np.clip(np.rint((1 - 2.0 * cw + sigma * rng.standard_normal(nn)) * 2 / sigma ** 2 * 3), -120,
                      120).astype(np.int8)
        llr[e:] = 0
        if f:
            llr[k - 2 * z - f:k - 2 * z] = 127
        n_in = nn if t % 4 else int(rng.integers(e, nn + 1)) // z * z  # also pass trimmed buffers
        n_in = max(n_in, k + 2 * z)
        cfg = LdpcDecoderConfiguration(bg, z, f, order, int(rng.integers(1, 16)))
        jobs.append(CodeblockJob(llr[:n_in], cfg, poly))
    return jobs


def test_random_mixed_batch_matches_port(batch_decoder, port):
    jobs = random_jobs(123, 160)
    outs, iters = batch_decoder.decode_batch(jobs)
    for j, o, it in zip(jobs, outs, iters):
        c = j.cfg
        p = -1 if j.crc_poly == 255 else j.crc_poly
        want_it, want_bits = port.ldpc_decode(c.base_graph, c.lifting_size, j.llrs, filler=c.nof_filler_bits,
                                              crc_poly=p, max_iter=c.max_iterations)
        k = golden_io.kbits(c.base_graph, c.lifting_size)
        assert it == want_it, (c, j.crc_poly)
        assert (unpack(o, k) == unpack(want_bits, k)).all(), (c, j.crc_poly)


def test_ldpc_batch_workload_matches_reference(batch_decoder, port):
    """The 512-codeblock BG1/BG2 Z=384 batch: every codeblock bit-exact, and every CRC-passing
    codeblock equals the transmitted bits."""
    b = sim.ldpc_batch(seed=0, n=512)
    outs, iters = batch_decoder.decode_batch(b.jobs)
    try:
        from oracle import REF_SO, Ref
        import os
        checker = Ref() if os.path.exists(REF_SO) else None
    except Exception:
        checker = None
    for i, (j, o, it) in enumerate(zip(b.jobs, outs, iters)):
        c = j.cfg
        k = golden_io.kbits(c.base_graph, c.lifting_size)
        if checker is not None:
            want_it, want_bits = checker.ldpc_decode(c.base_graph, c.lifting_size, j.llrs, max_iter=c.max_iterations)
        else:
            want_it, want_bits = port.ldpc_decode(c.base_graph, c.lifting_size, j.llrs, max_iter=c.max_iterations)
        assert it == want_it, i
        assert (unpack(o, k) == unpack(want_bits, k)).all(), i
        if it > 0:
            assert (unpack(o, k) == b.truth[i]).all()


def test_single_decoder_interface(batch_decoder):
    """LdpcDecoder.decode keeps the reference's contract: optional iteration count."""
    dec = LdpcDecoder(batch=batch_decoder)
    for c in golden_io.ldpc_cases():
        if c["poly"] == 255:
            crc = None
        else:
            crc = CrcCalculator(c["poly"])
        out = np.zeros(output_bytes(c["bg"], c["z"]), np.uint8)
        cfg = job_for(c).cfg
        res = dec.decode(out, c["llrs"], crc, cfg)
        assert (res or 0) == c["iterations"]


def test_device_entry_matches_host(batch_decoder):
    import torch
    jobs = random_jobs(7, 40)
    outs, iters = batch_decoder.decode_batch(jobs)
    descs, llrs, nbytes = make_descriptors(jobs)
    d_llrs = torch.from_numpy(llrs).cuda()
    d_bits = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(len(jobs), dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    batch_decoder.decode_device(descs, len(jobs), d_llrs.data_ptr(), d_bits.data_ptr(), d_it.data_ptr(),
                                stream.cuda_stream)
    stream.synchronize()
    assert (d_it.cpu().numpy() == iters).all()
    host_bits = np.concatenate(outs)
    assert (d_bits.cpu().numpy() == host_bits).all()


def test_invalid_descriptors_rejected(batch_decoder):
    cfg = LdpcDecoderConfiguration(1, 17, 0, 24, 6)  # 17 is not a lifting size
    with pytest.raises(_native.PgError) as e:
        batch_decoder.decode_batch([CodeblockJob(np.ones(66 * 17, np.int8), cfg, 2)])
    assert e.value.code == _native.PG_ERR_INVALID
    cfg = LdpcDecoderConfiguration(1, 16, 0, 24, 6)
    with pytest.raises(_native.PgError):
        batch_decoder.decode_batch([CodeblockJob(np.ones(10, np.int8), cfg, 2)])  # too few LLRs
    cfg = LdpcDecoderConfiguration(1, 16, 0, 24, 0)
    with pytest.raises(_native.PgError):
        batch_decoder.decode_batch([CodeblockJob(np.ones(66 * 16, np.int8), cfg, 2)])  # zero iterations


def test_capacity_rejected(ctx):
    from pusch_b200.ldpc import LdpcBatchDecoder
    small = LdpcBatchDecoder(max_codeblocks=2)
    cfg = LdpcDecoderConfiguration(2, 8, 0, 24, 4)
    jobs = [CodeblockJob(np.ones(50 * 8, np.int8), cfg, 2)] * 3
    with pytest.raises(_native.PgError) as e:
        small.decode_batch(jobs)
    assert e.value.code == _native.PG_ERR_CAPACITY
    small.ctx.close()


def test_pair_mode_saturation_and_short_inputs_match_port(batch_decoder, port):
    """Lifting sizes above 192 (the pair mode of the two-lanes-per-thread decoder) at high SNR, where
    soft bits saturate to +-127 and the infinity rules decide, with fillers, every CRC and trimmed or
    too-short inputs."""
    rng = np.random.default_rng(384)
    jobs = []
    for t in range(64):
        bg = 1 + (t & 1)
        z = [384, 208, 224, 240, 256, 288, 320, 352][(t >> 1) % 8]
        k = golden_io.kbits(bg, z)
        nn = (66 if bg == 1 else 50) * z
        poly = [0, 1, 2, 255][t % 4]
        cpoly = 2 if poly == 255 else poly
        order = 16 if cpoly == 0 else 24
        f = int(rng.integers(0, 400)) if t % 3 else 0
        msg = np.concatenate([codec.attach_crc(cpoly, rng.integers(0, 2, k - f - order, dtype=np.uint8)),
                              np.zeros(f, np.uint8)])
        cw = codec.ldpc_encode(bg, z, msg)
        snr_db = rng.uniform(4, 12) if t % 5 else rng.uniform(-1, 2)
        sigma = np.sqrt(1 / (2 * 10 ** (snr_db / 10)))
        llr = np.clip(np.rint((1 - 2.0 * cw + sigma * rng.standard_normal(nn)) * 2 / sigma ** 2 * 4), -120,
                      120).astype(np.int8)
        if f:
            llr[k - 2 * z - f:k - 2 * z] = 127
        e = int(rng.integers(k + 2 * z, nn + 1)) if t % 7 else k  # the last ones: fewer LLRs than message bits
        llr[e:] = 0
        cfg = LdpcDecoderConfiguration(bg, z, f, order, int(rng.integers(1, 12)))
        jobs.append(CodeblockJob(llr, cfg, poly))
    outs, iters = batch_decoder.decode_batch(jobs)
    for j, o, it in zip(jobs, outs, iters):
        c = j.cfg
        p = -1 if j.crc_poly == 255 else j.crc_poly
        want_it, want_bits = port.ldpc_decode(c.base_graph, c.lifting_size, j.llrs, filler=c.nof_filler_bits,
                                              crc_poly=p, max_iter=c.max_iterations)
        k = golden_io.kbits(c.base_graph, c.lifting_size)
        assert it == want_it, (c, j.crc_poly)
        assert (unpack(o, k) == unpack(want_bits, k)).all(), (c, j.crc_poly)


@pytest.mark.parametrize("kernel", [_native.PG_LDPC_KERNEL_ONE_LANE, _native.PG_LDPC_KERNEL_TWO_LANES,
                                    _native.PG_LDPC_KERNEL_SPLIT, _native.PG_LDPC_KERNEL_Z384,
                                    _native.PG_LDPC_KERNEL_Z384_SPLIT])
def test_every_kernel_bit_exact(batch_decoder, port, kernel):
    """The five decoding kernels (one lane per thread; two lanes per thread; two lanes per thread
    pair with the rows split over the pair; the Z = 384 specialisation, with one or two threads per
    lane pair) on the golden cases, a random
    mixed batch of 19 lifting sizes and the 512-codeblock BG1/BG2 Z=384 batch: bits and iteration
    counts equal the reference's and the restatement's."""
    batch_decoder.set_kernel(kernel)
    try:
        cases = golden_io.ldpc_cases()
        outs, iters = batch_decoder.decode_batch([job_for(c) for c in cases])
        for c, o, it in zip(cases, outs, iters):
            k = golden_io.kbits(c["bg"], c["z"])
            assert it == c["iterations"], (kernel, c["bg"], c["z"], c["poly"])
            assert (unpack(o, k) == unpack(c["bits"], k)).all(), (kernel, c["bg"], c["z"])
        jobs = random_jobs(55, 96) + sim.ldpc_batch(seed=3, n=512).jobs
        outs, iters = batch_decoder.decode_batch(jobs)
        for i, (j, o, it) in enumerate(zip(jobs, outs, iters)):
            c = j.cfg
            p = -1 if j.crc_poly == 255 else j.crc_poly
            want_it, want_bits = port.ldpc_decode(c.base_graph, c.lifting_size, j.llrs, filler=c.nof_filler_bits,
                                                  crc_poly=p, max_iter=c.max_iterations)
            k = golden_io.kbits(c.base_graph, c.lifting_size)
            assert it == want_it, (kernel, i)
            assert (unpack(o, k) == unpack(want_bits, k)).all(), (kernel, i)
    finally:
        batch_decoder.set_kernel(_native.PG_LDPC_KERNEL_SPLIT)
