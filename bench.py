#!/usr/bin/env python3
"""Benchmark of the B200 PUSCH receive path: the LDPC decoder batch workload.

Workload (one "step"): decode one batch of 512 codeblocks - BG1 Z=384 (K=8448, E=N=25344, rate
1/3) and BG2 Z=384 (K=3840, E=N=19200, rate 1/5) mixed 50/50 by seed - of random bits with
CRC24B, BPSK over AWGN at Eb/N0 ~ U[1, 3] dB, int8 LLRs saturated at +-127, at most 10
iterations with CRC early stop. The metric is decoded information Gbit/s (K - 24 bits of every
CRC-passing codeblock per second).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Our arm prints one JSON line with the device-timed value (inputs resident in HBM, one kernel
launch per step, L2 flushed between steps), the end-to-end value through the host C ABI
(pg_ldpc_decode_batch_host: pinned host LLRs in, bits and iteration counts out, every step),
the integer-ALU roofline of the decoding kernel, clocks sampled during the timed region and the
reference CPU decoder timed on this host. ``--impl reference`` times the reference's own CPU
LDPC decoder (oracle/_ref, AVX-512/AVX2) on all host cores on the same workload.
Under torchrun each rank decodes its own batch (seed + rank): weak scaling, no data-path
collective; rank 0 reports the aggregate over the max per-rank time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ocudu-dapp-platform_b200"))

METRIC = "PUSCH Mbit/s/B200 batched+learned vs plain GPU at BLER≤10%; LDPC Gbit/s"
N_CBS = 512
WORKLOAD = ("LDPC decoder batch: 512 codeblocks, BG1 Z=384 (K=8448, rate 1/3) and BG2 Z=384 (K=3840, rate 1/5) "
            "mixed 50/50 by seed, CRC24B, BPSK/AWGN Eb/N0 U[1,3] dB, int8 LLRs (scale 4/LLR unit, sat +-127), "
            "max 10 iterations, CRC early stop")
INT_OPS_PER_EDGE = 10  # algorithmic integer operations per edge update


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample length")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.rows = []
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200", "-i",
                 str(gpu_index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def wait_first_sample(self, timeout=3.0):
        """Blocks until the sampler has produced a row, so the timed region is covered."""
        t0 = time.time()
        while self.proc is not None and not self.rows and time.time() - t0 < timeout:
            time.sleep(0.02)

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


def edges_in_rows(bg, nof_rows):
    from pusch_b200 import codec
    deg, _, _ = codec.base_graph(bg)
    return int(deg[:nof_rows].sum())


def workload_stats(batch, iters):
    """Info bits of passing codeblocks, all codeblocks, and algorithmic integer ops executed."""
    import numpy as np
    bits_ok = int(sum(int(b) for b, it in zip(batch.info_bits, iters) if it > 0))
    bits_all = int(np.sum(batch.info_bits))
    ops = 0
    edge_updates = 0
    for j, it in zip(batch.jobs, iters):
        c = j.cfg
        k = (22 if c.base_graph == 1 else 10) * c.lifting_size
        # Rows processed: all check rows covered by the (full-buffer) input.
        n_in = int(np.max(np.nonzero(j.llrs)[0]) + 1) if np.any(j.llrs) else 0
        cb_len = max(n_in + 2 * c.lifting_size, k + 4 * c.lifting_size)
        cb_len = -(-cb_len // c.lifting_size) * c.lifting_size
        rows = min(cb_len // c.lifting_size - (22 if c.base_graph == 1 else 10), 46 if c.base_graph == 1 else 42)
        runs = int(it) if it > 0 else c.max_iterations
        e = runs * edges_in_rows(c.base_graph, rows) * c.lifting_size
        edge_updates += e
        ops += e * INT_OPS_PER_EDGE
    return bits_ok, bits_all, ops, edge_updates


def cpu_reference_decode(batch, seconds, cores, min_batches=1):
    """Decodes the batch with the reference's CPU decoder (oracle/_ref) on `cores` C++ threads,
    one reference decoder per thread with codeblocks claimed dynamically, until `seconds` of
    decoding have been timed (at least min_batches full batches). Returns (passing info bits,
    timed seconds, codeblocks, decoder variant)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Ref  # CPU baseline only
    ref = Ref()
    jobs = batch.jobs
    meta = np.array([[j.cfg.base_graph, j.cfg.lifting_size, j.cfg.nof_filler_bits, j.crc_poly, j.cfg.max_iterations,
                      j.llrs.size] for j in jobs], np.int32)
    offs = np.cumsum([0] + [j.llrs.size for j in jobs])[:-1]
    llrs = np.concatenate([j.llrs for j in jobs])
    info = np.asarray(batch.info_bits)
    bits, done, total, nb = 0, 0, 0.0, 0
    while True:
        it, dt = ref.ldpc_decode_batch_mt(meta, offs, llrs, cores)
        total += dt
        bits += int(info[it > 0].sum())
        done += len(jobs)
        nb += 1
        if nb >= min_batches and total >= seconds:
            break
    return bits, total, done, ref.variant


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from pusch_b200 import sim
    batch = sim.ldpc_batch(seed=args.seed, n=N_CBS)
    cores = host_cores()
    # Warm-up steps, then K timed steps; each step decodes the whole batch on all host cores.
    cpu_reference_decode(batch, 0.0, cores, min_batches=max(args.warmup, 1))
    times, bits = [], 0
    for _ in range(args.steps):
        b, dt, _, variant = cpu_reference_decode(batch, 0.0, cores, min_batches=1)
        times.append(dt)
        bits = b  # identical every step (deterministic decoder)
    ms = 1e3 * statistics.mean(times)
    value = bits / (ms * 1e-3) / 1e9
    line = {
        "metric": METRIC, "value": round(value, 4), "unit": "Gbit/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8", "data": "synthetic (seeded simulator)", "impl": "reference",
        "config": {"workload": WORKLOAD, "codeblocks_per_step": N_CBS},
        "cpu_baseline": {"value": round(value, 4), "unit": "Gbit/s", "cores": cores, "kind": "reference",
                         "sample": f"full 512-codeblock batch per step, reference ldpc_decoder_{variant} "
                                   f"(oracle/_ref) on {cores} C++ threads, one decoder per thread"},
        "e2e": {"value": round(value, 4), "unit": "Gbit/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local_rank = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    from pusch_b200 import sim
    from pusch_b200.ldpc import LdpcBatchDecoder, make_descriptors

    batch = sim.ldpc_batch(seed=args.seed + rank, n=N_CBS)
    descs, llrs, nbytes = make_descriptors(batch.jobs)
    dec = LdpcBatchDecoder(device=dev, max_codeblocks=N_CBS)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    # Device-resident work list: descriptors, LLRs and outputs in HBM.
    import ctypes
    d_descs = torch.from_numpy(np.frombuffer(bytes(descs), dtype=np.uint8).copy()).cuda()
    d_llrs = torch.from_numpy(llrs).cuda()
    d_bits = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    d_it = torch.zeros(N_CBS, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def step():
        dec.decode_resident(d_descs.data_ptr(), N_CBS, d_llrs.data_ptr(), d_bits.data_ptr(), d_it.data_ptr(), sptr)

    for _ in range(args.warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    clocks = ClockSampler(dev)
    clocks.wait_first_sample()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        evs[k][0].record(stream)
        step()
        evs[k][1].record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    ms = statistics.mean(kernel_ms)
    iters = d_it.cpu().numpy()
    bits_ok, bits_all, ops, edge_updates = workload_stats(batch, iters)

    if world > 1:
        t = torch.tensor([ms], device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_max = float(t.item())
        b = torch.tensor([bits_ok], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(b)
        total_bits = float(b.item())
    else:
        ms_max, total_bits = ms, float(bits_ok)
    value = total_bits / (ms_max * 1e-3) / 1e9

    # End to end through the host C ABI: pinned LLRs in, bits + iterations out, every step.
    e2e = None
    if not args.no_e2e:
        h_llrs = torch.from_numpy(llrs).pin_memory()
        h_bits = torch.zeros(nbytes, dtype=torch.uint8).pin_memory()
        h_it = torch.zeros(N_CBS, dtype=torch.int32).pin_memory()

        def e2e_step():
            rc = dec.lib.pg_ldpc_decode_batch_host(dec.ctx.handle, ctypes.addressof(descs), N_CBS,
                                                   h_llrs.data_ptr(), h_llrs.numel(), h_bits.data_ptr(),
                                                   h_bits.numel(), h_it.data_ptr())
            dec.ctx.check(rc)

        for _ in range(max(args.warmup, 1)):
            e2e_step()
        et = []
        for _ in range(args.steps):
            flush.fill_(3)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            et.append(time.perf_counter() - t0)
        assert (h_it.numpy() == iters).all()
        e_ms = 1e3 * statistics.mean(et)
        if world > 1:
            t = torch.tensor([e_ms], device="cuda")
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e_ms = float(t.item())
        e2e = {"value": round(total_bits / (e_ms * 1e-3) / 1e9, 4), "unit": "Gbit/s",
               "h2d_bytes_per_step": int(h_llrs.numel() + len(bytes(descs))),
               "d2h_bytes_per_step": int(h_bits.numel() + 4 * N_CBS), "ms_per_step": round(e_ms, 3)}

    # Integer roofline of the decoding kernel. Denominator: the measured full-rate integer
    # instruction throughput of this GPU (best of add.s32 / min.s32 in libpg_probe.so).
    peak_ops, classes = None, None
    try:
        probe = ctypes.CDLL(os.path.join(ROOT, "ocudu-dapp-platform_b200", "pusch_b200", "_lib", "libpg_probe.so"))
        probe.pg_probe_inst_classes.argtypes = [ctypes.c_int, ctypes.c_void_p]
        buf = (ctypes.c_double * 8)()
        if probe.pg_probe_inst_classes(dev, buf) == 0:
            names = ["add.s32", "min.s32", "mad.lo.u32", "prmt.b32", "min.s16x2", "add.f16x2", "min.f16x2",
                     "fma.f16x2"]
            classes = {n: round(buf[i] / 1e12, 2) for i, n in enumerate(names)}
            peak_ops = max(buf[0], buf[1])
    except OSError:
        pass
    achieved = ops / (ms * 1e-3) / 1e12
    props = torch.cuda.get_device_properties(dev)
    nominal = props.multi_processor_count * 128 * (clk["sm_max_mhz"] or 1965.0) * 1e6 / 1e12
    peak = peak_ops / 1e12 if peak_ops else nominal
    roofline = {
        "bound": "int", "kernel": "ldpc_decode_kernel", "achieved": round(achieved, 3), "peak": round(peak, 3),
        "unit": "Tops/s", "frac": round(achieved / peak, 4),
        "peak_source": ("measured: full-rate int32 instruction throughput (add.s32/min.s32 probe, libpg_probe.so)"
                        if peak_ops else "nominal 148 SM x 128 lanes x max SM clock"),
        "nominal_peak": round(nominal, 3), "instruction_classes_tops": classes,
        "ops_per_edge_update": INT_OPS_PER_EDGE, "edge_updates_per_launch": edge_updates,
        # dram__bytes_read.sum + dram__bytes_write.sum of one launch of this workload (ncu capture
        # summarised in profiles/ldpc_decode_kernel_ldpc-batch-512cb.md).
        "traffic": 17298000,
        "hbm_bytes_per_launch": int(llrs.size + nbytes + 4 * N_CBS + 20 * N_CBS),
    }

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        b, dt, ncb, variant = cpu_reference_decode(batch, args.cpu_seconds, cores)
        cpu = {"value": round(b / dt / 1e9, 4), "unit": "Gbit/s", "cores": cores, "kind": "reference",
               "sample": f"{ncb} codeblocks ({ncb // N_CBS} passes over the batch) with the reference "
                         f"ldpc_decoder_{variant} (oracle/_ref) on {cores} C++ threads, {dt:.1f} s"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "Gbit/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8", "data": "synthetic (seeded simulator)",
            "config": {"workload": WORKLOAD, "codeblocks_per_step": N_CBS * world,
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas{world}",
                       "info_bits_all_per_rank": bits_all, "info_bits_passing_per_rank": bits_ok,
                       "crc_pass": int((iters > 0).sum()), "mean_iterations": round(float(iters[iters > 0].mean()), 3)},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": args.steps,
            "kernel_ms": {"min": round(min(kernel_ms), 4), "max": round(max(kernel_ms), 4)},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    dec.ctx.close()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
