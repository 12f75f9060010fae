#!/usr/bin/env python3
"""Benchmark of the B200 PUSCH receive path.

Default workload (one "step"): the batched uneven slot - 16 cells of 100 MHz / 273 PRB, each with
1-16 UEs on contiguous PRB allocations, QPSK-256QAM (MCS table 2), 1-2 layers, 4 rx ports,
per-UE SNR U[0, 30] dB with link adaptation to BLER <= 10 %, DM-RS type 1 at symbols 2 and 11,
exponential-PDP channels (100 ns RMS, 8 taps), max 6 LDPC iterations - decoded through one slot
plan: DM-RS estimation, the learned channel estimator's refinement (committed parameters),
demodulation, rate dematching, LDPC, TB assembly and CRC; one CUDA graph replayed per step, launch
shapes picked by the plan's autotuner. The metric is decoded Mbit/s: the TBS of every UE whose TB
CRC passes (and equals the transmitted bits), per second of device time, inputs resident in HBM,
L2 flushed between steps.

The line also carries: the same plan with the plain estimator (batched_plain); the plain per-UE
GPU path on the same slot (one plan per UE, executed one after another with the host waiting for
each UE's result); the end-to-end value through the host entry (pg_pusch_plan_execute_host: pinned
host grids in, TBs and results out, every step); the rooflines of the learned estimator's network
(tensor cores) and of ldpc_decode_kernel (integer pipe), both timed with CUDA events inside the
step; the LDPC decoder batch (512 codeblocks, BG1/BG2 Z=384) in Gbit/s; clocks sampled during the
timed region; and the reference's CPU receive path (oracle/_ref, the reference's own stage objects)
on this host's cores as cpu_baseline.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload uneven|ldpc] [--no-learned]

``--impl reference`` times the reference's CPU receive path on all host cores on the same
workload. Under torchrun each rank decodes its own slot (seed + rank): weak scaling, no data-path
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
N_CELLS = 16
MAX_ITER = 6
PUSCH_WORKLOAD = ("Batched uneven slot: 16 cells x 273 PRB (100 MHz, 30 kHz SCS), 1-16 UEs per cell on contiguous "
                  "PRB allocations, QPSK-256QAM (MCS table 2) with link adaptation to BLER<=10%, 1-2 layers, 4 rx, "
                  "per-UE SNR U[0,30] dB, DM-RS type 1 symbols {2,11}, exponential PDP (100 ns RMS, 8 taps), "
                  "max 6 LDPC iterations, CRC early stop")
LE_FLOPS_PER_ROW = 2 * 5 * (16 * 64 + 12 * 64 * 64 + 64 * 16)  # 14 layers, kernel 5, per subcarrier row
WORKLOAD = ("LDPC decoder batch: 512 codeblocks, BG1 Z=384 (K=8448, rate 1/3) and BG2 Z=384 (K=3840, rate 1/5) "
            "mixed 50/50 by seed, CRC24B, BPSK/AWGN Eb/N0 U[1,3] dB, int8 LLRs (scale 4/LLR unit, sat +-127), "
            "max 10 iterations, CRC early stop")
# Algorithmic integer operations per edge update: v2c saturating subtraction, infinity guard, abs,
# three for the min1/min2 update, sign XOR, two for the message select and sign, promotion add.
INT_OPS_PER_EDGE = 10
LDPC_KERNEL_NAMES = ["ldpc_decode_kernel (one lifted lane per thread)",
                     "ldpc_decode_x2_kernel (two lifted lanes per thread for even Z > 192)",
                     "ldpc_decode_split_kernel (two lanes per thread pair, row edges split over the pair)",
                     "ldpc_decode_z_kernel (two lifted lanes per thread, Z = 384 specialised, f16 soft-bit pairs)",
                     "ldpc_decode_zs_kernel (Z = 384 specialised, row edges split over a thread pair)"]
# ncu figures of one launch of the LDPC batch per kernel (pg_ldpc_kernel id): DRAM bytes read +
# written, and pipe utilisation in % of active cycles. Kernel 1 at four CTAs per SM, kernel 3 at
# two (the bench default).
LDPC_NCU = {
    1: {"traffic": 24246528, "pipes": {"alu": 55.5, "fma": 32.3, "lsu": 24.9, "issue_active": 59.6,
                                       "sm_active_pct_of_elapsed": 60.4}},
    3: {"traffic": 11546880, "pipes": {"alu": 50.3, "issue_active": 53.3, "sm_active_pct_of_elapsed": 81.0}},
}
# Integer-instruction throughput probe (the LDPC roofline denominator), built by
# ocudu-dapp-platform_b200/measure/Makefile.
PROBE_SO = os.path.join(ROOT, "ocudu-dapp-platform_b200", "measure", "_lib", "libpg_probe.so")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="uneven", choices=["uneven", "ldpc"])
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample length")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--e2e-depth", type=int, default=3, choices=(1, 2, 3),
                   help="slots in flight in the pipelined end-to-end run (pg_pusch_plan_submit_host)")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--no-ldpc", action="store_true")
    p.add_argument("--no-learned", action="store_true", help="plain estimator only")
    p.add_argument("--no-autotune", action="store_true", help="default launch shapes (no autotuning run)")
    p.add_argument("--no-configs", action="store_true", help="skip the single-slot configuration sub-lines")
    p.add_argument("--learned-min-qm", type=int, default=6,
                   help="refine the UEs of this modulation order and above with the learned estimator (0: every UE)")
    p.add_argument("--ldpc-kernel", type=int, default=None,
                   help="LDPC batch kernel of the --workload ldpc line (pg_ldpc_kernel; default: the library's)")
    p.add_argument("--ldpc-ctas-per-sm", type=int, default=2,
                   help="resident LDPC CTAs per SM of the --workload ldpc line (0: the kernel limit)")
    p.add_argument("--ldpc-order", default="longest", choices=["given", "longest"],
                   help="work order of the --workload ldpc line's persistent decoders (pg_set_ldpc_order)")
    return p.parse_args()


def plan_kernels(plan):
    """Kernels one execution of the plan launches with its current tuning and estimator
    (pg_pusch_plan_info's count)."""
    import ctypes
    from pusch_b200._native import PgPuschPlanInfo
    info = PgPuschPlanInfo()
    plan.ctx.check(plan.lib.pg_pusch_plan_info(plan.handle, ctypes.byref(info)))
    return int(info.nof_kernels)


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


def pusch_edge_updates(ues, results):
    """Algorithmic LDPC edge updates of one slot: per codeblock, the check rows its input covers
    (trailing-zero trimming of the dematched buffer: E + F significant positions at rv 0) times
    the row edges times Z, times the UE's iterations run (failed codeblocks count the maximum)."""
    from pusch_b200 import codec
    from pusch_b200.sch import segment
    from pusch_b200.sim import nof_ch_symbols
    total = 0
    for ue, r in zip(ues, results):
        g = nof_ch_symbols(ue) * ue.modulation_order
        sg = segment(ue.tbs_bits, ue.base_graph, ue.modulation_order, ue.nof_layers, g // ue.modulation_order)
        z, kb = sg["lifting_size"], (22 if ue.base_graph == 1 else 10)
        n = (66 if ue.base_graph == 1 else 50) * z
        deg, _, _ = codec.base_graph(ue.base_graph)
        edges = 0
        for c in range(sg["nof_cbs"]):
            e = sg["e_short"] if c < sg["nof_short_cbs"] else sg["e_long"]
            n_in = min(e + sg["nof_filler_bits"], n)
            cb_len = max(n_in + 2 * z, kb * z + 4 * z)
            cb_len = -(-cb_len // z) * z
            rows = min(cb_len // z - kb, 46 if ue.base_graph == 1 else 42)
            edges += int(deg[:rows].sum()) * z
        total += edges * r.mean_iterations
    return int(total)


def bf16_peak():
    """Dense bf16 tensor peak (TFLOP/s) measured on this pool (MEASURED_PEAKS.json, burst figure),
    else the pool's earlier measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured (MEASURED_PEAKS.json bf16_tflops, burst)"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback (1.59 PFLOP/s earlier measurement on this pool)"


def hbm_peak():
    """Measured HBM copy bandwidth (GB/s, MEASURED_PEAKS.json), else the pool's earlier measurement."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def int_peak(dev):
    """Measured full-rate int32 instruction throughput (ops/s) of this GPU and the per-class
    figures (libpg_probe.so), or (None, None)."""
    import ctypes
    try:
        probe = ctypes.CDLL(PROBE_SO)
        probe.pg_probe_inst_classes.argtypes = [ctypes.c_int, ctypes.c_void_p]
        buf = (ctypes.c_double * 8)()
        if probe.pg_probe_inst_classes(dev, buf) == 0:
            names = ["add.s32", "min.s32", "mad.lo.u32", "prmt.b32", "min.s16x2", "add.f16x2", "min.f16x2",
                     "fma.f16x2"]
            return max(buf[0], buf[1]), {n: round(buf[i] / 1e12, 2) for i, n in enumerate(names)}
    except OSError:
        pass
    return None, None


SUB_CONFIGS = {
    "c1_20mhz_single_ue": ("Plain single-UE slot: 20 MHz / 30 kHz, 51 PRB, DM-RS symbol 2, 1 layer, 2 rx, QPSK "
                           "(MCS table 1 index 5, TBS 5888), flat Rayleigh, 10 dB, max 6 LDPC iterations"),
    "c3_100mhz_full_cell": ("Plain full-cell slot: 100 MHz / 30 kHz, 273 PRB, DM-RS symbols 2 and 11, 2 layers, 4 rx, "
                            "256QAM (MCS table 2 index 20, TBS 417976, 50 codeblocks), exponential PDP (100 ns RMS, "
                            "8 taps), 25 dB, max 6 LDPC iterations"),
}


def sub_config_lines(ctx, seed, steps, warmup, with_cpu, autotune=True):
    """The two single-slot configurations as sub-lines of the PUSCH line: one slot plan each (plain
    estimator, CUDA graph), device time per slot with CUDA events (L2 flushed between slots), decoded
    Mbit/s and slots/s; with the CPU baseline, the reference's CPU receive path on one thread on the
    same slot (Mbit/s) and whether its per-UE CRC flags, mean iterations and TBs equal the plan's."""
    import ctypes

    import numpy as np
    import torch

    from pusch_b200 import sim
    from pusch_b200._native import PgSchResult
    from pusch_b200.pusch import PuschSlotPlan, results_from

    out = {}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    for name, slot in (("c1_20mhz_single_ue", sim.single_ue_slot(seed=seed)),
                       ("c3_100mhz_full_cell", sim.full_cell_slot(seed=seed))):
        plan = PuschSlotPlan(ctx, [slot], max_iterations=MAX_ITER, graph=True)
        n = plan.n
        d_grid = torch.from_numpy(plan.grid.view(np.int32)).cuda()
        d_tb = torch.zeros(max(plan.tb_bytes, 1), dtype=torch.uint8, device="cuda")
        d_res = torch.zeros(n * ctypes.sizeof(PgSchResult), dtype=torch.uint8, device="cuda")
        if autotune:
            plan.autotune(d_grid.data_ptr(), reps=3)
        with torch.cuda.stream(stream):
            for _ in range(max(warmup, 3)):
                flush.fill_(1)
                plan.execute_device(d_grid.data_ptr(), d_tb.data_ptr(), d_res.data_ptr(), None, stream.cuda_stream)
            torch.cuda.synchronize()
            ts = []
            for k in range(steps):
                flush.fill_(k & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                plan.execute_device(d_grid.data_ptr(), d_tb.data_ptr(), d_res.data_ptr(), None, stream.cuda_stream)
                b.record(stream)
                stream.synchronize()
                ts.append(a.elapsed_time(b))
        res_arr = (PgSchResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
        res = results_from(plan.descs, res_arr, None, d_tb.cpu().numpy())
        good = [r.tb_crc_ok and bool((np.unpackbits(r.transport_block) == t).all()) for r, t in zip(res, slot.truth)]
        bits = int(sum(u.tbs_bits for u, g in zip(plan.ues, good) if g))
        ms = statistics.mean(ts)
        line = {"workload": SUB_CONFIGS[name], "value": round(bits / (ms * 1e-3) / 1e6, 3), "unit": "Mbit/s",
                "slots_per_s": round(1e3 / ms, 1), "ms_per_slot": round(ms, 4), "codeblocks": int(plan.info.nof_codeblocks),
                "bler": round(1.0 - sum(good) / n, 4), "estimator": "plain", "launch_shapes": plan.tuning().as_dict()}
        if with_cpu:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            from oracle import Ref  # CPU baseline and parity flags only
            ref = Ref()
            descs = plan.descs
            r = ref.pusch_decode_detail(descs, plan.grid, plan.tb_bytes, int(plan.info.nof_llrs), 1)
            same = all(g.tb_crc_ok == bool(o) and g.mean_iterations == float(it) and
                       (not g.tb_crc_ok or np.array_equal(g.transport_block,
                                                          r["tb"][d.tb_out_offset:d.tb_out_offset + d.tbs_bits // 8]))
                       for g, o, it, d in zip(res, r["ok"], r["mean_iters"], descs))
            total, passes = 0.0, 0
            while total < 2.0 or passes < 3:
                ok, _, _, dt = ref.pusch_decode_mt(descs, plan.grid, plan.tb_bytes, 1)
                total += dt
                passes += 1
            ref_bits = int(sum(u.tbs_bits for u, o in zip(plan.ues, ok) if o))
            line["reference_matches"] = bool(same)
            line["cpu_baseline"] = {"value": round(ref_bits * passes / total / 1e6, 3), "unit": "Mbit/s", "cores": 1,
                                    "kind": "reference",
                                    "sample": f"{passes} passes over the slot through the reference's CPU stage objects "
                                              f"(oracle/_ref) on 1 thread, {total:.2f} s"}
        out[name] = line
        plan.close()
    return out


def reference_pusch(slots, seconds, cores, min_passes=1):
    """The reference's CPU receive path (oracle/_ref: the reference's own stage objects, one UE
    per thread) over the whole slot until `seconds` of decoding are timed. Returns (decoded bits
    of the last pass, timed seconds, passes, UEs per pass)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Ref  # CPU baseline only
    from pusch_b200.pusch import batch_descriptors
    ref = Ref()
    descs, grid, tb_bytes, ues = batch_descriptors(slots, max_iterations=MAX_ITER)
    total, passes, bits = 0.0, 0, 0
    while True:
        ok, _, _, dt = ref.pusch_decode_mt(descs, grid, tb_bytes, cores)
        total += dt
        passes += 1
        bits = int(sum(u.tbs_bits for u, o in zip(ues, ok) if o))
        if passes >= min_passes and total >= seconds:
            break
    return bits, total, passes, len(ues)


def run_reference_pusch(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    slots = pusch_workload(args.seed)
    cores = host_cores()
    reference_pusch(slots, 0.0, cores, min_passes=max(args.warmup, 1))
    times, bits, n_ues = [], 0, 0
    for _ in range(args.steps):
        b, dt, _, n_ues = reference_pusch(slots, 0.0, cores, min_passes=1)
        times.append(dt)
        bits = b
    ms = 1e3 * statistics.mean(times)
    value = bits / (ms * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mbit/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32/int8", "data": "synthetic (seeded simulator)", "impl": "reference",
        "config": pusch_config(slots, args.gpus, args.seed),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mbit/s", "cores": cores, "kind": "reference",
                         "sample": f"the full {N_CELLS}-cell slot ({n_ues} UEs) per step through the reference's CPU "
                                   f"stage objects (oracle/_ref) on {cores} C++ threads, one UE per thread at a time"},
        "e2e": {"value": round(value, 3), "unit": "Mbit/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def pusch_workload(seed):
    from pusch_b200 import sim
    return sim.uneven_cells(seed=seed, nof_cells=N_CELLS)


def pusch_config(slots, world, seed):
    """The workload keys of the PUSCH line, identical in both arms: computed from the simulated
    slots with the simulator's own (transmit-side) segmentation, so the reference arm needs no
    part of the GPU library."""
    from pusch_b200 import codec
    from pusch_b200.sim import nof_ch_symbols
    ues = [u for sl in slots for u in sl.ues]
    cbs = sum(codec.segment_tx(u.tbs_bits, u.base_graph, u.modulation_order, u.nof_layers,
                               nof_ch_symbols(u))["nof_cbs"] for u in ues)
    return {"workload": PUSCH_WORKLOAD, "cells_per_rank": len(slots), "ues_per_rank": len(ues),
            "codeblocks_per_rank": int(cbs), "tb_bits_per_rank": int(sum(u.tbs_bits for u in ues)),
            "seed": seed, "max_iterations": MAX_ITER, "parallelism": f"replicas{world}"}


def run_ours_pusch(args):
    import ctypes

    import numpy as np
    import torch

    rank, world, dev = dist_setup()

    from pusch_b200 import _native
    from pusch_b200._native import PgSchResult
    from pusch_b200.pusch import PuschSlotPlan, results_from

    from pusch_b200 import learned as le_mod

    slots = pusch_workload(args.seed + rank)
    config = pusch_config(slots, world, args.seed)
    truth = [t for sl in slots for t in sl.truth]
    ctx = _native.Context(device=dev, max_codeblocks=64)
    plan = PuschSlotPlan(ctx, slots, max_iterations=MAX_ITER, graph=True)
    n = plan.n
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    d_grid = torch.from_numpy(plan.grid.view(np.int32)).cuda()
    d_tb = torch.zeros(max(plan.tb_bytes, 1), dtype=torch.uint8, device="cuda")
    d_res = torch.zeros(n * ctypes.sizeof(PgSchResult), dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    # The learned estimator (trained parameters committed with the package) refines the channel
    # estimates of the UEs at 64QAM and 256QAM inside the plan (--learned-min-qm): its evaluation
    # (python -m pusch_b200.learned evaluate --min-qm 6) gives the same BLER and goodput as refining
    # every UE from 12 dB up, and the same goodput below. Without parameters the plan runs the plain
    # estimator.
    params = None if args.no_learned else le_mod.load_params()
    le_use = [ue.modulation_order >= args.learned_min_qm for ue in plan.ues]
    le_rows = plan.le_rows(le_use)
    net = le_mod.LearnedEstimator(ctx, max_rows=max(le_rows, 1), params=params) if params is not None else None

    def step():
        plan.execute_device(d_grid.data_ptr(), d_tb.data_ptr(), d_res.data_ptr(), None, sptr)

    def decoded():
        """Decoded bits: CRC-passing UEs whose TB equals the transmitted bits."""
        res_arr = (PgSchResult * n).from_buffer_copy(d_res.cpu().numpy().tobytes())
        res = results_from(plan.descs, res_arr, None, d_tb.cpu().numpy())
        ok = [r.tb_crc_ok and bool((np.unpackbits(r.transport_block) == t).all()) for r, t in zip(res, truth)]
        return res, ok, int(sum(u.tbs_bits for u, g in zip(plan.ues, ok) if g))

    def timed(nsteps, sample_clocks=False):
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                flush.fill_(1)
                step()
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        clocks = ClockSampler(dev) if sample_clocks else None
        if clocks is not None:
            clocks.wait_first_sample()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(nsteps)]
        k_ms, l_ms = [], []
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for k in range(nsteps):
                flush.fill_(k & 0xFF)
                evs[k][0].record(stream)
                step()
                evs[k][1].record(stream)
                stream.synchronize()
                k_ms.append(ctx.lib.pg_last_kernel_ms(ctx.handle))
                l_ms.append(ctx.lib.pg_last_learned_ms(ctx.handle))
        torch.cuda.synchronize()
        clk = clocks.stop() if clocks is not None else None
        return [a.elapsed_time(b) for a, b in evs], k_ms, l_ms, clk

    # Launch shapes picked by the autotuner on this slot (with the estimator that is timed next).
    if net is not None:
        plan.set_learned(net, use=le_use)
    tuning = plan.tuning() if args.no_autotune else plan.autotune(d_grid.data_ptr(), reps=5)[0]
    if net is not None:
        plan.set_learned(None)
    ctx.lib.pg_set_kernel_timing(ctx.handle, 1)
    # Batched path with the plain estimator (the comparison point of the learned one).
    batched_plain = None
    if net is not None:
        p_step_ms, _, _, _ = timed(max(10, min(args.steps, 200)))
        _, p_ok, p_bits = decoded()
        p_ms = statistics.mean(p_step_ms)
        batched_plain = {"value": round(p_bits / (p_ms * 1e-3) / 1e6, 3), "unit": "Mbit/s", "ms_per_step": round(p_ms, 4),
                         "bler": round(1.0 - sum(p_ok) / n, 4),
                         "what": "the same slot plan with the plain estimator (LS + RC FIR + linear interpolation)"}
        plan.set_learned(net, use=le_use)
    step_ms, ldpc_ms, learned_ms, clk = timed(args.steps, sample_clocks=True)
    ms = statistics.mean(step_ms)
    results, good, bits_ok = decoded()
    bits_all = int(sum(u.tbs_bits for u in plan.ues))
    bler = 1.0 - sum(good) / n

    ms_max, total_bits = max_over_ranks(ms, world), sum_over_ranks(bits_ok, world)
    value = total_bits / (ms_max * 1e-3) / 1e6

    # Plain per-UE GPU path: one plan per UE, each executed and waited for before the next UE.
    plain = None
    if not args.no_plain:
        per_ue = []
        for sl in slots:
            for u in range(len(sl.ues)):
                one = type(sl)(sl.grid, [sl.ues[u]], [sl.truth[u]], sl.nof_ports, sl.nof_prb_grid, sl.slot,
                               sl.scs_khz, sl.dmrs_scaling)
                per_ue.append(PuschSlotPlan(ctx, [one], max_iterations=MAX_ITER, graph=False))
        grids = [torch.from_numpy(p.grid.view(np.int32)).cuda() for p in per_ue]
        tbs = [torch.zeros(max(p.tb_bytes, 1), dtype=torch.uint8, device="cuda") for p in per_ue]
        res1 = torch.zeros(ctypes.sizeof(PgSchResult), dtype=torch.uint8, device="cuda")

        def plain_step():
            for p, g, tb in zip(per_ue, grids, tbs):
                p.execute_device(g.data_ptr(), tb.data_ptr(), res1.data_ptr(), None, sptr)
                stream.synchronize()

        with torch.cuda.stream(stream):
            for _ in range(max(1, args.warmup)):
                plain_step()
            pms = []
            for k in range(max(3, min(20, args.steps // 5))):
                flush.fill_(k & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                plain_step()
                b.record(stream)
                torch.cuda.synchronize()
                pms.append(a.elapsed_time(b))
        p_ms = statistics.mean(pms)
        # The per-UE plans decode what the batched plan with the plain estimator decodes.
        plain_bits = bits_ok if batched_plain is None else p_bits
        plain = {"value": round(plain_bits / (p_ms * 1e-3) / 1e6, 3), "unit": "Mbit/s", "ms_per_step": round(p_ms, 3),
                 "plans": len(per_ue), "kernels_per_step": sum(plan_kernels(p) for p in per_ue),
                 "what": "one plan per UE executed in turn, host waits for each UE's result (no batching, no graph)"}
        for p in per_ue:
            p.close()

    # End to end through the host entry: pinned grids in, results and TBs out, every step.
    e2e = None
    if not args.no_e2e:
        h_grid = torch.from_numpy(plan.grid.view(np.int32)).pin_memory()
        h_tb = torch.zeros(max(plan.tb_bytes, 1), dtype=torch.uint8).pin_memory()
        h_res = (PgSchResult * n)()
        lib = ctx.lib

        def e2e_step():
            ctx.check(lib.pg_pusch_plan_execute_host(plan.handle, h_grid.data_ptr(), h_tb.data_ptr(), h_tb.numel(),
                                                     ctypes.addressof(h_res), None))

        for _ in range(max(args.warmup, 1)):
            e2e_step()
        et = []
        for k in range(min(args.steps, 200)):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            et.append(time.perf_counter() - t0)
        e_ms = 1e3 * statistics.mean(et)
        e_ok = [bool(h_res[i].tb_crc_ok) for i in range(n)]
        assert e_ok == [r.tb_crc_ok for r in results]
        e_ms = max_over_ranks(e_ms, world)
        e2e = {"value": round(total_bits / (e_ms * 1e-3) / 1e6, 3), "unit": "Mbit/s",
               "h2d_bytes_per_step": int(plan.info.h2d_grid_bytes),
               "d2h_bytes_per_step": int(plan.tb_bytes + n * ctypes.sizeof(PgSchResult)),
               "ms_per_step": round(e_ms, 3), "entry": "pg_pusch_plan_execute_host"}

        # Consecutive slots through the pipelined entries: each step's grids still go host to
        # device and its results device to host, but the copy of slot k + 1 overlaps slot k.
        def pipelined(steps, depth=3):
            t0 = time.perf_counter()
            for k in range(steps):
                ctx.check(lib.pg_pusch_plan_submit_host(plan.handle, h_grid.data_ptr()))
                if k >= depth - 1:
                    ctx.check(lib.pg_pusch_plan_collect_host(plan.handle, h_tb.data_ptr(), h_tb.numel(),
                                                             ctypes.addressof(h_res), None))
            for _ in range(min(steps, depth - 1)):
                ctx.check(lib.pg_pusch_plan_collect_host(plan.handle, h_tb.data_ptr(), h_tb.numel(),
                                                         ctypes.addressof(h_res), None))
            return time.perf_counter() - t0

        pipelined(max(args.warmup, 2), args.e2e_depth)
        np_steps = min(args.steps, 200)
        p_ms = 1e3 * pipelined(np_steps, args.e2e_depth) / np_steps
        assert [bool(h_res[i].tb_crc_ok) for i in range(n)] == [r.tb_crc_ok for r in results]
        p_ms = max_over_ranks(p_ms, world)
        # The headline end-to-end figure is the pipelined one (consecutive slots, as a PHY runs them);
        # the one-call-at-a-time figure stays beside it.
        e2e = {"value": round(total_bits / (p_ms * 1e-3) / 1e6, 3), "unit": "Mbit/s",
               "h2d_bytes_per_step": int(plan.info.h2d_grid_bytes),
               "d2h_bytes_per_step": int(plan.tb_bytes + n * ctypes.sizeof(PgSchResult)),
               "ms_per_step": round(p_ms, 3),
               "slots_in_flight": args.e2e_depth,
               "entry": "pg_pusch_plan_submit_host / pg_pusch_plan_collect_host (slots in flight as above; every step "
                        "copies its grids in and its results out)",
               "synchronous": e2e}

        # The same through the Open Fronthaul payload: the grids as 9-bit BFP PRBs (the radio
        # unit's gain of 1/16 into the fixed-point range and its compression, done here by the
        # simulator), decompressed on the GPU.
        from pusch_b200 import sim as sim_mod
        h_comp = torch.from_numpy(sim_mod.bfp_compress(sim_mod.scale_grid_words(plan.grid.ravel(), 1.0 / 16),
                                                       9)).pin_memory()

        def bfp_step():
            ctx.check(lib.pg_pusch_plan_execute_host_bfp(plan.handle, h_comp.data_ptr(), h_comp.numel(), 9,
                                                         h_tb.data_ptr(), h_tb.numel(), ctypes.addressof(h_res), None))

        for _ in range(max(args.warmup, 1)):
            bfp_step()
        bt = []
        for k in range(min(args.steps, 200)):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            bfp_step()
            bt.append(time.perf_counter() - t0)
        b_ms = 1e3 * statistics.mean(bt)
        tbh = h_tb.numpy()
        b_bits = 0
        for i, d in enumerate(plan.descs):
            if h_res[i].tb_crc_ok and (np.unpackbits(tbh[d.tb_out_offset:d.tb_out_offset + d.tbs_bits // 8])
                                       == truth[i]).all():
                b_bits += d.tbs_bits
        b_ms = max_over_ranks(b_ms, world)
        e2e["ofh_bfp9"] = {"value": round(b_bits / (b_ms * 1e-3) / 1e6, 3), "unit": "Mbit/s",
                           "h2d_bytes_per_step": int(h_comp.numel()),
                           "d2h_bytes_per_step": int(plan.tb_bytes + n * ctypes.sizeof(PgSchResult)),
                           "ms_per_step": round(b_ms, 3), "decoded_bits": int(b_bits),
                           "entry": "pg_pusch_plan_execute_host_bfp (9-bit BFP grids, decompressed on the GPU)"}

    # Rooflines: the integer pipe of ldpc_decode_kernel and the tensor cores of the learned
    # estimator's convolutions, both timed with CUDA events inside the step; "roofline" is the one
    # that takes the larger share of the step.
    edge_updates = pusch_edge_updates(plan.ues, results)
    ops = edge_updates * INT_OPS_PER_EDGE
    valid_ms = [x for x in ldpc_ms if x > 0]
    k_ms = statistics.mean(valid_ms) if valid_ms else float("nan")
    peak_ops, classes = int_peak(dev)
    props = torch.cuda.get_device_properties(dev)
    nominal = props.multi_processor_count * 128 * (clk["sm_max_mhz"] or 1965.0) * 1e6 / 1e12
    peak = peak_ops / 1e12 if peak_ops else nominal
    achieved = ops / (k_ms * 1e-3) / 1e12
    roofline = {
        "bound": "int",
        "kernel": LDPC_KERNEL_NAMES[tuning.as_dict().get("ldpc_kernel", 0)],
        "achieved": round(achieved, 3), "peak": round(peak, 3),
        "unit": "Tops/s", "frac": round(achieved / peak, 4),
        "peak_source": ("measured: full-rate int32 instruction throughput (add.s32/min.s32 probe, libpg_probe.so)"
                        if peak_ops else "nominal 148 SM x 128 lanes x max SM clock"),
        "nominal_peak": round(nominal, 3), "instruction_classes_tops": classes,
        "ops_per_edge_update": INT_OPS_PER_EDGE, "edge_updates_per_launch": edge_updates,
        "kernel_ms": round(k_ms, 4), "kernel_share_of_step": round(k_ms / ms, 3),
        "traffic": None,
    }

    rooflines = {"ldpc": roofline}
    le_ms = statistics.mean([x for x in learned_ms if x > 0]) if net is not None else float("nan")
    if net is not None:
        flops = le_rows * LE_FLOPS_PER_ROW
        peak_tf, peak_src = bf16_peak()
        ach = flops / (le_ms * 1e-3) / 1e12
        rooflines["learned"] = {
            "bound": "tensor", "kernel": "le_fused_forward_kernel (14 layers in one launch) + le_features/le_apply",
            "achieved": round(ach, 2), "peak": peak_tf, "unit": "TFLOP/s", "frac": round(ach / peak_tf, 4),
            "peak_source": peak_src, "flops_per_launch_chain": flops, "rows": le_rows,
            "flops_per_row": LE_FLOPS_PER_ROW, "stage_ms": round(le_ms, 4), "stage_share_of_step": round(le_ms / ms, 3),
            "traffic": None}
        if le_ms > k_ms:
            roofline = rooflines["learned"]

    ldpc_line = None
    if not args.no_ldpc:
        ldpc_line = ldpc_measure(args, dev, rank, world)
    uci_line = uci_measure(ctx, plan.ues, hbm_peak()) if rank == 0 else None
    bfp_line = bfp_measure(ctx, plan.grid.ravel(), hbm_peak()) if rank == 0 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        b, dt, passes, n_ues = reference_pusch(slots, args.cpu_seconds, cores)
        cpu = {"value": round(b * passes / dt / 1e6, 3), "unit": "Mbit/s", "cores": cores, "kind": "reference",
               "sample": f"{passes} passes over the full {N_CELLS}-cell slot ({n_ues} UEs) through the reference's "
                         f"CPU stage objects (oracle/_ref) on {cores} C++ threads, {dt:.1f} s"}
        b1, dt1, passes1, _ = reference_pusch(slots, max(2.0, args.cpu_seconds / 4), 1)
        cpu["one_thread"] = {"value": round(b1 * passes1 / dt1 / 1e6, 3), "unit": "Mbit/s", "cores": 1,
                             "sample": f"{passes1} passes over the same slot on 1 thread, {dt1:.1f} s"}
    sub_lines = sub_config_lines(ctx, args.seed + rank, max(10, min(args.steps, 100)), args.warmup,
                                 rank == 0 and world == 1 and not args.no_cpu_baseline,
                                 not args.no_autotune) if rank == 0 and not args.no_configs else None

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mbit/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32/int8", "data": "synthetic (seeded simulator)",
            "config": config,
            "run": {"decoded_bits_per_rank": bits_ok, "bler": round(bler, 4),
                    "l2": "flushed between steps (256 MiB write)", "graph": "one CUDA graph per step",
                    "launch_shapes": tuning.as_dict(),
                    "estimator": ("learned (residual 1-D CNN, 6 blocks x 64 ch, k=5, BF16 tensor cores; DM-RS "
                                  "corrections and time-basis terms over the slot) on the plain LS + RC FIR + "
                                  "linear interpolation" if net is not None else
                                  "plain (LS + RC FIR + linear interpolation)"),
                    "learned_ues": (f"modulation order >= {args.learned_min_qm}: {sum(le_use)} of {n} UEs, "
                                    f"{le_rows} estimator rows" if net is not None else None)},
            "slots_per_s": round(1e3 / ms_max * world, 1),
            "configs": sub_lines,
            "plain_per_ue": plain, "batched_plain": batched_plain,
            "e2e": e2e, "roofline": roofline, "rooflines": rooflines, "ldpc": ldpc_line, "uci": uci_line, "ofh_bfp": bfp_line, "cpu_baseline": cpu,
            "clocks": clk,
            "gpu_launches": plan_kernels(plan) * args.steps,
            "step_ms": {"min": round(min(step_ms), 4), "max": round(max(step_ms), 4)},
        }
        print(json.dumps(line), flush=True)
    plan.close()
    if net is not None:
        net.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    ctx.close()
    return 0


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


def ldpc_core(args, dev, rank, world, with_cpu=True, with_e2e=True, steps=None):
    """The LDPC decoder batch (512 codeblocks) on this rank's GPU; returns rank 0's JSON line."""
    import numpy as np
    import torch

    steps = steps or args.steps

    from pusch_b200 import sim
    from pusch_b200.ldpc import LdpcBatchDecoder, make_descriptors

    batch = sim.ldpc_batch(seed=args.seed + rank, n=N_CBS)
    descs, llrs, nbytes = make_descriptors(batch.jobs)
    dec = LdpcBatchDecoder(device=dev, max_codeblocks=N_CBS)
    if args.ldpc_kernel is not None:
        dec.set_kernel(args.ldpc_kernel)
    dec.set_ctas_per_sm(args.ldpc_ctas_per_sm)
    dec.set_order(0 if args.ldpc_order == "given" else 1)
    kernel_id = args.ldpc_kernel if args.ldpc_kernel is not None else int(dec.ctx.lib.pg_get_ldpc_kernel(dec.ctx.handle))
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
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for k in range(steps):
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

    ms_max, total_bits = max_over_ranks(ms, world), sum_over_ranks(bits_ok, world)
    value = total_bits / (ms_max * 1e-3) / 1e9

    # End to end through the host C ABI: pinned LLRs in, bits + iterations out, every step.
    e2e = None
    if with_e2e and not args.no_e2e:
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
        for _ in range(steps):
            flush.fill_(3)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            e2e_step()
            et.append(time.perf_counter() - t0)
        assert (h_it.numpy() == iters).all()
        e_ms = 1e3 * statistics.mean(et)
        e_ms = max_over_ranks(e_ms, world)
        e2e = {"value": round(total_bits / (e_ms * 1e-3) / 1e9, 4), "unit": "Gbit/s",
               "h2d_bytes_per_step": int(h_llrs.numel() + len(bytes(descs))),
               "d2h_bytes_per_step": int(h_bits.numel() + 4 * N_CBS), "ms_per_step": round(e_ms, 3)}

    # Integer roofline of the decoding kernel. Denominator: the measured full-rate integer
    # instruction throughput of this GPU (best of add.s32 / min.s32 in libpg_probe.so).
    peak_ops, classes = None, None
    try:
        probe = ctypes.CDLL(PROBE_SO)
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
        "bound": "int",
        "kernel": LDPC_KERNEL_NAMES[kernel_id] + " (every codeblock of the batch has Z=384)",
        "ctas_per_sm": args.ldpc_ctas_per_sm or "kernel limit",
        "achieved": round(achieved, 3), "peak": round(peak, 3),
        "unit": "Tops/s", "frac": round(achieved / peak, 4),
        "peak_source": ("measured: full-rate int32 instruction throughput (add.s32/min.s32 probe, libpg_probe.so)"
                        if peak_ops else "nominal 148 SM x 128 lanes x max SM clock"),
        "nominal_peak": round(nominal, 3), "instruction_classes_tops": classes,
        "ops_per_edge_update": INT_OPS_PER_EDGE, "edge_updates_per_launch": edge_updates,
        # dram__bytes_read.sum + dram__bytes_write.sum of one launch on this workload, and the pipe
        # utilisation, for the kernels with an ncu capture (summarised in
        # profiles/ldpc_decode_kernel_ldpc-batch-512cb.md); null for the others.
        "traffic": LDPC_NCU.get(kernel_id, {}).get("traffic"),
        "ncu_pipes_pct_of_active": LDPC_NCU.get(kernel_id, {}).get("pipes"),
        "hbm_bytes_per_launch": int(llrs.size + nbytes + 4 * N_CBS + 20 * N_CBS),
    }

    cpu = None
    if with_cpu and rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = host_cores()
        b, dt, ncb, variant = cpu_reference_decode(batch, args.cpu_seconds, cores)
        cpu = {"value": round(b / dt / 1e9, 4), "unit": "Gbit/s", "cores": cores, "kind": "reference",
               "sample": f"{ncb} codeblocks ({ncb // N_CBS} passes over the batch) with the reference "
                         f"ldpc_decoder_{variant} (oracle/_ref) on {cores} C++ threads, {dt:.1f} s"}

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "Gbit/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int8", "data": "synthetic (seeded simulator)",
            "config": {"workload": WORKLOAD, "codeblocks_per_step": N_CBS * world,
                       "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas{world}",
                       "info_bits_all_per_rank": bits_all, "info_bits_passing_per_rank": bits_ok,
                       "crc_pass": int((iters > 0).sum()), "mean_iterations": round(float(iters[iters > 0].mean()), 3)},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk, "gpu_launches": steps,
            "kernel_ms": {"min": round(min(kernel_ms), 4), "max": round(max(kernel_ms), 4)},
        }
    dec.ctx.close()
    return line


def max_over_ranks(x, world, device="cuda"):
    """The largest x over the ranks (times are taken as the slowest rank's)."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x, world, device="cuda"):
    """The sum of x over the ranks (work done by the whole job)."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t)
    return float(t.item())


def dist_setup():
    import torch
    rank, world, local_rank = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    return rank, world, torch.cuda.current_device()


def run_ours_ldpc(args):
    import torch
    rank, world, dev = dist_setup()
    line = ldpc_core(args, dev, rank, world)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def uci_measure(ctx, ues, peak_gbs):
    """UCI on PUSCH for every UE of the slot: HARQ-ACK of 5 bits and CSI Part 1 of 8 bits on each
    codeword (demultiplexed out of synthetic descrambled soft bits of the slot's codeword sizes),
    then short-block detection of the 2 x UEs messages; CUDA-event time of both entries, and the
    demultiplexer against the measured HBM bandwidth (it reads and writes every soft bit once)."""
    import ctypes
    import torch
    from pusch_b200._native import PgUciShortBlock
    from pusch_b200.sim import nof_ch_symbols
    from pusch_b200.uci import make_config
    cfgs, offs, in_off = [], [0, 0, 0], 0
    lib = ctx.lib
    for ue in ues:
        bpr = ue.modulation_order * ue.nof_layers
        g = nof_ch_symbols(ue) * ue.modulation_order
        mask = sum(1 << s for s in ue.dmrs_symbols)
        c = make_config(nof_llrs=g, c_init=(ue.rnti << 15) + ue.n_id_data, nof_prb=ue.nof_rb, dmrs_symbol_mask=mask,
                        modulation_order=ue.modulation_order, nof_layers=ue.nof_layers, start_symbol_index=0,
                        nof_symbols=14, dmrs_type=1, nof_cdm_groups_without_data=2, nof_harq_ack_bits=5,
                        nof_csi_part1_bits=8, nof_enc_harq_ack_bits=bpr * max(3, 24 // bpr),
                        nof_enc_csi_part1_bits=bpr * max(4, 48 // bpr))
        sz = (ctypes.c_uint32 * 3)()
        if lib.pg_ulsch_demultiplex_sizes(ctypes.byref(c), sz):
            continue
        c.llr_offset, c.sch_offset, c.harq_ack_offset, c.csi_part1_offset = in_off, offs[0], offs[1], offs[2]
        in_off += g
        offs = [offs[k] + sz[k] for k in range(3)]
        cfgs.append((c, tuple(sz)))
    if not cfgs:
        return None
    n = len(cfgs)
    arr = (type(cfgs[0][0]) * n)(*[c for c, _ in cfgs])
    gen = torch.Generator(device="cuda").manual_seed(5)
    d_in = torch.randint(-120, 121, (in_off,), dtype=torch.int8, device="cuda", generator=gen)
    outs = [torch.zeros(max(1, offs[k]), dtype=torch.int8, device="cuda") for k in range(3)]
    items = (PgUciShortBlock * (2 * n))()
    for i, (c, sz) in enumerate(cfgs):
        for j, (off, e, k) in enumerate(((c.harq_ack_offset, sz[1], 5), (offs[1] + c.csi_part1_offset, sz[2], 8))):
            it = items[2 * i + j]
            it.llr_offset, it.nof_llrs, it.out_offset = off, e, (2 * i + j) * 8
            it.nof_bits, it.modulation_order = k, c.modulation_order
    uci_in = torch.zeros(max(1, offs[1] + offs[2]), dtype=torch.int8, device="cuda")
    d_bits = torch.zeros(16 * n, dtype=torch.uint8, device="cuda")
    d_valid = torch.zeros(2 * n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()

    def demux():
        ctx.check(lib.pg_ulsch_demultiplex_device(ctx.handle, ctypes.addressof(arr), n, d_in.data_ptr(),
                                                  outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                                  st.cuda_stream))

    def detect():
        ctx.check(lib.pg_uci_short_block_detect_device(ctx.handle, ctypes.addressof(items), 2 * n, uci_in.data_ptr(),
                                                       d_bits.data_ptr(), d_valid.data_ptr(), st.cuda_stream))

    demux()
    torch.cuda.synchronize()
    uci_in[:offs[1]] = outs[1][:offs[1]]
    uci_in[offs[1]:offs[1] + offs[2]] = outs[2][:offs[2]]
    times, kernel = {}, {}
    lib.pg_set_kernel_timing(ctx.handle, 1)
    for name, fn in (("demux", demux), ("detect", detect)):
        for _ in range(3):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        ks = []
        for a, b in ev:
            a.record(st)
            fn()
            b.record(st)
            b.synchronize()
            ks.append(float(lib.pg_last_kernel_ms(ctx.handle)))
        times[name] = statistics.mean(a.elapsed_time(b) for a, b in ev)
        kernel[name] = statistics.mean(ks)
    # Polar-coded CSI Part 1: one 100-bit message of 400 soft bits per UE (CRC11, N = 512 with
    # puncturing), synthetic soft bits.
    from pusch_b200._native import PgUciPolar
    pol = (PgUciPolar * n)()
    for i in range(n):
        pol[i].llr_offset, pol[i].nof_llrs, pol[i].out_offset, pol[i].nof_bits = 400 * i, 400, 100 * i, 100
    p_in = torch.randint(-120, 121, (400 * n,), dtype=torch.int8, device="cuda", generator=gen)
    p_bits = torch.zeros(100 * n, dtype=torch.uint8, device="cuda")

    def polar():
        ctx.check(lib.pg_uci_polar_decode_device(ctx.handle, ctypes.addressof(pol), n, p_in.data_ptr(),
                                                 p_bits.data_ptr(), d_valid.data_ptr(), st.cuda_stream))

    for name, fn in (("polar", polar),):
        for _ in range(3):
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(20)]
        ks = []
        for a, b in ev:
            a.record(st)
            fn()
            b.record(st)
            b.synchronize()
            ks.append(float(lib.pg_last_kernel_ms(ctx.handle)))
        times[name] = statistics.mean(a.elapsed_time(b) for a, b in ev)
        kernel[name] = statistics.mean(ks)
    gbs = 2 * in_off / (kernel["demux"] * 1e-3) / 1e9
    return {"ues": n, "harq_ack_bits": 5, "csi_part1_bits": 8, "soft_bits": int(in_off),
            "polar": {"messages": n, "bits": 100, "soft_bits_per_message": 400, "kernel_ms": round(kernel["polar"], 4),
                      "call_ms": round(times["polar"], 4),
                      "note": "one CTA per message, one warp per codeblock; latency-bound (sequential SC tree walk)"},
            "call_ms": {k: round(v, 4) for k, v in times.items() if k != "polar"},
            "demux_kernel_ms": round(kernel["demux"], 4), "detect_kernel_ms": round(kernel["detect"], 4),
            "demux_roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak_gbs, "unit": "GB/s",
                               "frac": round(gbs / peak_gbs, 4), "bytes_per_launch": int(2 * in_off)},
            "data": "synthetic descrambled soft bits of the slot's codeword sizes, L2 not flushed between launches"}


def bfp_measure(ctx, grid_words, peak_gbs):
    """Open Fronthaul BFP decompression of the slot's grids (9-bit PRBs, the radio unit's gain of
    1/16 and compression done by the simulator): kernel time through the context's kernel events
    and the HBM roofline (compressed bytes read + complex bf16 words written, per launch)."""
    import torch
    from pusch_b200 import sim as sim_mod
    comp = sim_mod.bfp_compress(sim_mod.scale_grid_words(grid_words, 1.0 / 16), 9)
    nprb = grid_words.size // 12
    d_in = torch.from_numpy(comp).cuda()
    d_out = torch.empty(12 * nprb, dtype=torch.int32, device="cuda")
    lib = ctx.lib
    st = torch.cuda.current_stream()
    lib.pg_set_kernel_timing(ctx.handle, 1)
    ks = []
    for k in range(23):
        ctx.check(lib.pg_bfp_decompress_device(ctx.handle, d_in.data_ptr(), nprb, 9, d_out.data_ptr(), st.cuda_stream))
        st.synchronize()
        if k >= 3:
            ks.append(float(lib.pg_last_kernel_ms(ctx.handle)))
    ms = statistics.mean(ks)
    nbytes = int(comp.size + 4 * 12 * nprb)
    gbs = nbytes / (ms * 1e-3) / 1e9
    return {"prbs": int(nprb), "data_width": 9, "kernel_ms": round(ms, 4),
            "roofline": {"bound": "hbm", "achieved": round(gbs, 1), "peak": peak_gbs, "unit": "GB/s",
                         "frac": round(gbs / peak_gbs, 4), "bytes_per_launch": nbytes}}


def ldpc_measure(args, dev, rank, world):
    """The LDPC batch as a sub-measurement of the PUSCH line (device-timed Gbit/s and roofline)."""
    line = ldpc_core(args, dev, rank, world, with_cpu=False, with_e2e=False, steps=min(args.steps, 100))
    if line is None:
        return None
    return {"value": line["value"], "unit": "Gbit/s", "ms_per_step": line["ms_per_step"],
            "workload": WORKLOAD, "roofline": {k: line["roofline"][k] for k in ("achieved", "peak", "unit", "frac")},
            "crc_pass": line["config"]["crc_pass"], "mean_iterations": line["config"]["mean_iterations"]}




def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference_pusch(args) if args.workload == "uneven" else run_reference(args)
    return run_ours_pusch(args) if args.workload == "uneven" else run_ours_ldpc(args)


if __name__ == "__main__":
    sys.exit(main())
