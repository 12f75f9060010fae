"""Learned channel estimator on the B200: host side of the pg_le_* entries (include/pusch_b200.h).

The network (csrc/learned_est.cu) refines the plain DM-RS estimator's frequency responses per
(UE, receive port, layer) allocation; training and inference run on the GPU through the library's
own tensor-core forward and backward kernels. This module holds the parameter initialisation,
a wrapper of one pg_le_net, the seeded training-data source (the project's PUSCH channel model,
evaluated on the GPU with torch as device-memory plumbing), the training loop and the evaluation
of BLER / EVM / channel-estimate error against the plain estimator.

There is no counterpart in the reference: its estimator is port_channel_estimator_average_impl
(lib/phy/upper/signal_processors/channel_estimator/port_channel_estimator_average_impl.cpp), which
stays the per-allocation fallback and the baseline every evaluation compares against.
"""
import ctypes
import functools
import math
import os
import time

import numpy as np

from . import _native, prg
from ._native import PgLeAdam
from .pusch import PgPortResult, PgPuschUe

LAYERS = [(16, 64)] + [(64, 64)] * 12 + [(64, 16)]
TAPS = 5
HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "le_weights.npz")
DMRS_SYMBOLS = (2, 11)
BETA = float(np.float32(10 ** (3 / 20)))


def nof_params():
    return sum(TAPS * ci * co + co for ci, co in LAYERS)


def init_params(seed=0):
    """He-normal weights, zero biases; the second layer of each residual block and the output
    layer start small, so that the untrained network adds almost nothing to the plain estimate."""
    rng = np.random.default_rng(seed)
    parts = []
    for i, (cin, cout) in enumerate(LAYERS):
        std = math.sqrt(2.0 / (TAPS * cin))
        if i == len(LAYERS) - 1:
            std *= 0.02
        elif i >= 2 and i % 2 == 0:
            std *= 0.1
        parts += [rng.standard_normal(TAPS * cin * cout) * std, np.zeros(cout)]
    return np.concatenate(parts).astype(np.float32)


class LearnedEstimator:
    """One pg_le_net: parameters, forward/backward on given features, refinement and training."""

    def __init__(self, ctx: _native.Context, max_rows: int, params=None):
        self.ctx = ctx
        self.lib = _native.load()
        self.max_rows = int(max_rows)
        h = ctypes.c_void_p()
        ctx.check(self.lib.pg_le_create(ctx.handle, self.max_rows, ctypes.byref(h)))
        self.handle = h
        self.n = int(self.lib.pg_le_nof_params())
        assert self.n == nof_params()
        self.set_params(init_params(0) if params is None else params)

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        self.ctx.check(self.lib.pg_le_set_params(self.handle, p.ctypes.data_as(ctypes.c_void_p), p.size))

    def params(self):
        p = np.zeros(self.n, np.float32)
        self.ctx.check(self.lib.pg_le_get_params(self.handle, p.ctypes.data_as(ctypes.c_void_p), p.size))
        return p

    def grads(self):
        g = np.zeros(self.n, np.float32)
        self.ctx.check(self.lib.pg_le_get_grads(self.handle, g.ctypes.data_as(ctypes.c_void_p), g.size))
        return g

    def status(self):
        self.ctx.check(self.lib.pg_le_status(self.handle))

    def forward(self, x_ptr, valid_ptr, rows, y_ptr, stream=0):
        self.ctx.check(self.lib.pg_le_forward_device(self.handle, x_ptr, valid_ptr, rows, y_ptr, stream))

    def backward(self, dy_ptr, rows, stream=0):
        self.ctx.check(self.lib.pg_le_backward_device(self.handle, dy_ptr, rows, stream))

    def refine(self, descs, ls_ptr, est_ptr, pr_ptr, use=None, basis_ptr=None, stream=0):
        """Corrects est in place; with basis_ptr (a buffer of est's size), writes the time-basis
        coefficients of the UEs with two DM-RS symbols there (pg_le_refine_device)."""
        n = len(descs)
        u = None if use is None else (ctypes.c_uint8 * n)(*[int(bool(v)) for v in use])
        self.ctx.check(self.lib.pg_le_refine_device(self.handle, ctypes.addressof(descs), n, ls_ptr, est_ptr,
                                                    basis_ptr, pr_ptr, u, stream))

    def train_step(self, descs, ls_ptr, est_ptr, pr_ptr, h_ptr, opt: PgLeAdam, loss_ptr, stream=0):
        self.ctx.check(self.lib.pg_le_train_step_device(self.handle, ctypes.addressof(descs), len(descs), ls_ptr,
                                                        est_ptr, pr_ptr, h_ptr, ctypes.byref(opt), loss_ptr,
                                                        stream))

    def save(self, path=WEIGHTS, **meta):
        np.savez_compressed(path, params=self.params(), **{k: np.asarray(v) for k, v in meta.items()})

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pg_le_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def load_params(path=WEIGHTS):
    """The trained parameters committed with the library (None when absent)."""
    if not os.path.exists(path):
        return None
    return np.load(path)["params"].astype(np.float32)


# ----------------------------------------------------------------------------------------------
# Training data: the simulator's channel model at the DM-RS symbols, on the GPU.

@functools.lru_cache(maxsize=4096)
def _pilots(slot, symbol, n_id):
    """Layer-0 DM-RS pilots of a 273-PRB allocation starting at PRB 0 (a prefix serves any
    allocation that starts at PRB 0)."""
    return prg.dmrs_type1(slot, symbol, n_id, 0, 273, 1)[0]


def cbf16_words(torch, re, im):
    """float32 tensors -> complex bf16 words (real in the low half, round to nearest even)."""
    r = re.to(torch.bfloat16).view(torch.int16).to(torch.int32) & 0xFFFF
    i = im.to(torch.bfloat16).view(torch.int16).to(torch.int32) & 0xFFFF
    return r | (i << 16)


class DmrsTrainingSource:
    """Seeded batches of UEs with DM-RS-only grids (symbols 2 and 11, 4 receive ports) and their
    true channel at all 14 OFDM symbols ([port][symbol][layer][12 nof_rb] per UE, the layout
    pg_le_train_step_device reads). Per UE: allocation
    1-273 PRB (half log-uniform, half uniform), 1 or 2 layers, SNR U[snr_db], exponential PDP of 8
    taps with RMS delay U[delay_ns], Rayleigh taps with Jakes' Doppler spectrum (16 sinusoids)
    at a maximum Doppler U[doppler_hz]."""

    def __init__(self, seed=0, nof_ports=4, snr_db=(0.0, 30.0), delay_ns=(30.0, 300.0), doppler_hz=(0.0, 500.0),
                 scs_khz=30, n_ids=8, device="cuda"):
        import torch
        self.torch = torch
        self.rng = np.random.default_rng(seed)
        self.gen = torch.Generator(device=device)
        self.gen.manual_seed(int(seed) + 12345)
        self.nof_ports, self.snr_db, self.delay_ns, self.doppler_hz = nof_ports, snr_db, delay_ns, doppler_hz
        self.scs = scs_khz * 1e3
        self.n_ids = n_ids
        self.device = device
        t = np.arange(14) * (1e-3 / (scs_khz / 15) / 14)
        self.t_sym = torch.tensor(t, dtype=torch.float32, device=device)

    def draw_ue(self):
        r = self.rng
        nrb = int(round(math.exp(r.uniform(0, math.log(273))))) if r.random() < 0.5 else int(r.integers(1, 274))
        return dict(nof_rb=max(1, min(273, nrb)), nof_layers=int(r.integers(1, 3)), snr=float(r.uniform(*self.snr_db)),
                    delay=float(r.uniform(*self.delay_ns)) * 1e-9, doppler=float(r.uniform(*self.doppler_hz)),
                    slot=int(r.integers(0, 20)), n_id=int(r.integers(0, self.n_ids)))

    def batch(self, rows):
        """UEs until about `rows` network rows; returns (descs, grid words, h_true, est size, params)."""
        torch = self.torch
        ues, total = [], 0
        while total < rows:
            u = self.draw_ue()
            total += self.nof_ports * u["nof_layers"] * (12 * u["nof_rb"] + 2)
            ues.append(u)
        return self.make(ues)

    def make(self, ues):
        torch = self.torch
        P = self.nof_ports
        descs = (PgPuschUe * len(ues))()
        grid_off, est_off = 0, 0
        grids, hs = [], []
        for i, u in enumerate(ues):
            K, L = 12 * u["nof_rb"], u["nof_layers"]
            d = descs[i]
            d.grid_offset, d.grid_nof_subc = grid_off, K
            d.est_offset = est_off
            d.llr_offset, d.tbs_bits, d.tb_out_offset, d.nref = 0, 0, 0, 0
            d.dmrs_scaling = BETA
            d.rb_start, d.nof_rb = 0, u["nof_rb"]
            d.dmrs_symbol_mask = sum(1 << s for s in DMRS_SYMBOLS)
            d.n_id, d.rnti, d.n_id_data, d.dc_subcarrier = u["n_id"], 1, 0, -1
            d.slot, d.n_scid, d.first_symbol, d.nof_symbols = u["slot"], 0, 0, 14
            d.nof_rx_ports, d.nof_layers, d.modulation_order = P, L, 2
            d.base_graph, d.rv, d.max_iterations = 1, 0, 1
            h = self.channel(u, K, L)                                  # [P][L][14][K] complex64
            g = torch.zeros((P, 14, K), dtype=torch.int32, device=self.device)
            nv = 10 ** (-u["snr"] / 10)
            for di, s in enumerate(DMRS_SYMBOLS):
                pil = torch.from_numpy(_pilots(u["slot"], s, u["n_id"])[:K // 2]).to(self.device)
                pl = pil.unsqueeze(0).repeat(L, 1)
                if L > 1:
                    pl[1, 1::2] *= -1
                rx = torch.zeros((P, K), dtype=torch.complex64, device=self.device)
                rx[:, 0::2] = (h[:, :, s, 0::2] * pl.unsqueeze(0)).sum(1) * BETA
                noise = torch.randn((2, P, K), generator=self.gen, device=self.device) * math.sqrt(nv / 2)
                g[:, s, :] = cbf16_words(torch, rx.real + noise[0], rx.imag + noise[1])
            grids.append(g.reshape(-1))
            hs.append(h.permute(0, 2, 1, 3).reshape(-1))            # [P][14][L][K]
            grid_off += P * 14 * K
            est_off += P * 2 * L * K
        grid = torch.cat(grids)
        h_true = torch.view_as_real(torch.cat(hs)).contiguous()
        return descs, grid, h_true, est_off, ues

    def channel(self, u, K, L):
        torch = self.torch
        P, T, M = self.nof_ports, 8, 16
        tau = torch.linspace(0, 3 * u["delay"], T, device=self.device)
        pw = torch.exp(-tau / u["delay"])
        pw = pw / pw.sum()
        f = torch.arange(K, device=self.device, dtype=torch.float32) * self.scs
        steer = torch.exp(-2j * math.pi * (tau[:, None] * f[None, :]).to(torch.complex64))          # [T][K]
        ang = torch.rand((P, L, T, M), generator=self.gen, device=self.device) * 2 * math.pi
        ph = torch.rand((P, L, T, M), generator=self.gen, device=self.device) * 2 * math.pi
        arg = 2 * math.pi * u["doppler"] * torch.cos(ang)[..., None] * self.t_sym + ph[..., None]    # [P][L][T][M][14]
        a = torch.exp(1j * arg.to(torch.complex64)).sum(3) / math.sqrt(M)                         # [P][L][T][14]
        a = a * torch.sqrt(pw)[None, None, :, None]
        return torch.einsum("pltd,tk->pldk", a, steer)


def train(ctx, steps=3000, rows_per_step=96_000, seed=0, lr=1e-3, lr_min=2e-5, log_every=100, params=None,
          time_budget_s=None, verbose=True):
    """Trains a network on the GPU; returns (LearnedEstimator, history of (step, net MSE, plain MSE))."""
    import torch
    src = DmrsTrainingSource(seed)
    net = LearnedEstimator(ctx, max_rows=rows_per_step + 4 * 2 * (12 * 273 + 2), params=params)
    lib = _native.load()
    loss = torch.zeros((log_every, 2), dtype=torch.float32, device="cuda")
    hist, t0 = [], time.time()
    stream = torch.cuda.current_stream().cuda_stream
    for it in range(steps):
        descs, grid, h_true, est_size, _ = src.batch(rows_per_step)
        n = len(descs)
        est = torch.empty(2 * est_size, dtype=torch.float32, device="cuda")
        ls = torch.empty_like(est)
        pr = torch.empty((n * 4, 5), dtype=torch.float32, device="cuda")
        ctx.check(lib.pg_pusch_estimate_ls_device(ctx.handle, ctypes.addressof(descs), n, grid.data_ptr(),
                                                  est.data_ptr(), ls.data_ptr(), pr.data_ptr(), stream))
        frac = it / max(1, steps - 1)
        opt = PgLeAdam(lr=lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * frac)), beta1=0.9, beta2=0.999,
                       eps=1e-8, weight_decay=0.0)
        net.train_step(descs, ls.data_ptr(), est.data_ptr(), pr.data_ptr(), h_true.data_ptr(), opt,
                       loss[it % log_every].data_ptr(), stream)
        if (it + 1) % log_every == 0 or it == steps - 1:
            m = loss[: (it % log_every) + 1].mean(0).cpu().numpy()
            hist.append((it + 1, float(m[0]), float(m[1])))
            if verbose:
                print(f"step {it + 1}: net MSE {m[0]:.5f} plain MSE {m[1]:.5f} ({time.time() - t0:.1f} s)", flush=True)
            if time_budget_s is not None and time.time() - t0 > time_budget_s:
                break
    net.status()
    return net, hist


# ----------------------------------------------------------------------------------------------
# Evaluation against the plain estimator.

EVAL_DELAY_NS = (30.0, 300.0)
EVAL_DOPPLER_HZ = (0.0, 500.0)
EVAL_MARGIN_STEP_DB = 1.0
EVAL_MARGIN_MAX_DB = 14.0
EVAL_BLER_TARGET = 0.1
SLOT_S = 0.5e-3


def eval_slots(snr_db, seed=0, cells=4, la_margin_db=4.0):
    """Uneven slots (sim.uneven_cells) with every UE at snr_db, RMS delay spread U[30, 300] ns and
    maximum Doppler U[0, 500] Hz; the link adaptation of sim.uneven_cells with its thresholds
    raised by la_margin_db (they are calibrated on 100 ns without Doppler)."""
    from . import sim
    return sim.uneven_cells(seed, nof_cells=cells, snr_range=(snr_db, snr_db), delay_range_ns=EVAL_DELAY_NS,
                            doppler_range_hz=EVAL_DOPPLER_HZ, la_margin_db=la_margin_db)


def tb_errors(results, truths):
    return [not (r.tb_crc_ok and bool((np.unpackbits(r.transport_block) == t).all())) for r, t in zip(results, truths)]


def cbf16_to_complex(words):
    """uint32/int32 complex bf16 words (numpy) -> complex64."""
    w = np.asarray(words).astype(np.uint32)
    re = (w << 16).view(np.float32)
    im = (w & 0xFFFF0000).view(np.float32)
    return re + 1j * im


def grid_estimates(ctx, descs, est, basis=None):
    """The channel estimate of every UE at all 14 OFDM symbols, as the demodulator uses it
    (pg_pusch_symbol_estimates_device: time interpolation between the DM-RS symbols, plus the
    time-basis terms when basis is given, rounded to bf16): one complex64 array per UE,
    [port][14][layer][12 nof_rb]."""
    import torch
    lib = _native.load()
    out = []
    for i in range(len(descs)):
        d = descs[i]
        P, L, K = d.nof_rx_ports, d.nof_layers, 12 * d.nof_rb
        sym = torch.empty((P, 14, L, K), dtype=torch.int32, device="cuda")
        bp = None if basis is None else basis.data_ptr() + 8 * d.est_offset
        ctx.check(lib.pg_pusch_symbol_estimates_device(ctx.handle, ctypes.byref(d), est.data_ptr() + 8 * d.est_offset,
                                                       bp, sym.data_ptr(), None))
        out.append(cbf16_to_complex(sym.cpu().numpy()))
    return out


def data_symbol_nmse(descs, grids, truths):
    """Normalised squared error of per-UE [port][14][layer][K] estimates against the true channel
    over the symbols that carry no DM-RS."""
    err = sig = 0.0
    for i, (g, t) in enumerate(zip(grids, truths)):
        mask = descs[i].dmrs_symbol_mask
        data = [s for s in range(14) if not (mask >> s) & 1]
        e = g[:, data] - t[:, data]
        err += float(np.sum(np.abs(e) ** 2))
        sig += float(np.sum(np.abs(t[:, data]) ** 2))
    return err / sig


def split_truth(descs, h_true):
    """h_true of DmrsTrainingSource.make (real pairs, UEs back to back) -> per-UE complex
    [port][14][layer][K] arrays."""
    h = h_true.cpu().numpy().view(np.complex64).reshape(-1)
    out, off = [], 0
    for i in range(len(descs)):
        d = descs[i]
        shape = (d.nof_rx_ports, 14, d.nof_layers, 12 * d.nof_rb)
        m = int(np.prod(shape))
        out.append(h[off:off + m].reshape(shape))
        off += m
    return out


def _true_channel(slot, u):
    h = slot.channels[u]                                        # [P][L][nsc] or [P][L][14][nsc]
    if h.ndim == 3:
        h = np.stack([h] * 14, axis=2)
    return h.transpose(0, 2, 1, 3)                              # [P][14][L][nsc]


def estimate_quality(ctx, slots, net=None, max_iterations=6):
    """EVM of the MMSE-equalised data symbols and NMSE of the channel estimate over the data
    symbols, with the plain estimates and (when net is given) the refined ones with their
    time-basis terms, through the library's stage entries: estimation
    (pg_pusch_estimate_ls_device), refinement (pg_le_refine_device), per-symbol estimates
    (pg_pusch_symbol_estimates_device) and equalisation (pg_equalize_device)."""
    import torch
    from .pusch import batch_descriptors
    lib = _native.load()
    descs, grid, _, ues = batch_descriptors(slots, max_iterations)
    n = len(ues)
    # One response buffer for every UE of every cell (the per-cell descriptors restart at 0).
    off = 0
    for i in range(n):
        descs[i].est_offset = off
        off += 4 * len(ues[i].dmrs_symbols) * ues[i].nof_layers * 12 * ues[i].nof_rb
    d_grid = torch.from_numpy(grid.view(np.int32)).cuda()
    est_size = off
    est = torch.empty(2 * est_size, dtype=torch.float32, device="cuda")
    ls = torch.empty_like(est)
    pr = torch.empty((4 * n, 5), dtype=torch.float32, device="cuda")
    ctx.check(lib.pg_pusch_estimate_ls_device(ctx.handle, ctypes.addressof(descs), n, d_grid.data_ptr(),
                                              est.data_ptr(), ls.data_ptr(), pr.data_ptr(), None))
    variants = {"plain": (est, None)}
    if net is not None:
        est_l = est.clone()
        basis = torch.zeros_like(est)
        net.refine(descs, ls.data_ptr(), est_l.data_ptr(), pr.data_ptr(), basis_ptr=basis.data_ptr())
        variants["learned"] = (est_l, basis)
    torch.cuda.synchronize()
    prh = pr.cpu().numpy().reshape(n, 4, 5)
    slot_of = [(si, u) for si, sl in enumerate(slots) for u in range(len(sl.ues))]
    truths = [_true_channel(slots[si], u) for si, u in slot_of]
    out = {}
    for name, (e, bas) in variants.items():
        err = sig = 0.0
        g_all = grid_estimates(ctx, descs, e, bas)
        for i in range(n):
            d, ue = descs[i], ues[i]
            sl = slots[slot_of[i][0]]
            P, L, K = d.nof_rx_ports, d.nof_layers, 12 * d.nof_rb
            data_syms = [s for s in range(14) if s not in ue.dmrs_symbols]
            g = d_grid[d.grid_offset:d.grid_offset + P * 14 * d.grid_nof_subc].view(P, 14, d.grid_nof_subc)
            y = g[:, data_syms, 12 * d.rb_start:12 * d.rb_start + K].reshape(P, -1).contiguous()
            words = torch.from_numpy(g_all[i].astype(np.complex64).view(np.float32).reshape(P, 14, L, K, 2))
            hh = cbf16_words(torch, words[..., 0], words[..., 1])[:, data_syms].permute(0, 2, 1, 3)
            hh = hh.reshape(P, L, -1).contiguous().cuda()
            nre = y.shape[1]
            eq = torch.empty((nre, L, 2), dtype=torch.float32, device="cuda")
            nv = torch.empty((nre, L), dtype=torch.float32, device="cuda")
            nvh = np.ascontiguousarray(prh[i, :P, 0], np.float32)
            ctx.check(lib.pg_equalize_device(ctx.handle, 1, nre, P, L, y.data_ptr(), hh.data_ptr(),
                                             nvh.ctypes.data_as(ctypes.c_void_p), 1.0, eq.data_ptr(), nv.data_ptr(),
                                             None))
            torch.cuda.synchronize()
            z = eq.cpu().numpy().view(np.complex64)[..., 0]
            x = sl.symbols[slot_of[i][1]]
            err += float(np.sum(np.abs(z - x) ** 2))
            sig += float(np.sum(np.abs(x) ** 2))
        out[name] = dict(evm=math.sqrt(err / sig), nmse=data_symbol_nmse(descs, g_all, truths))
    return out


def learned_use(slots, min_qm=0):
    """Per UE of the slots: True where the learned refinement applies (modulation order at least
    min_qm; 0: every UE)."""
    return [ue.modulation_order >= min_qm for sl in slots for ue in sl.ues]


def run_plan(ctx, slots, net, max_iterations, min_qm=0):
    """(TB error flags, decoded bits) of every UE of the slots through a slot plan, with the plain
    estimator (net None) or the learned one (for the UEs of modulation order min_qm and above)."""
    from .pusch import PuschSlotPlan
    truths = [t for sl in slots for t in sl.truth]
    plan = PuschSlotPlan(ctx, slots, max_iterations=max_iterations)
    if net is not None:
        plan.set_learned(net, use=None if min_qm <= 0 else learned_use(slots, min_qm))
    err = tb_errors(plan.execute_host(), truths)
    if net is not None:
        plan.set_learned(None)
    plan.close()
    bits = sum(len(t) for t, e in zip(truths, err) if not e)
    return err, bits


def la_point(per_margin, key):
    """Outer-loop link adaptation: the smallest margin whose BLER is at most EVAL_BLER_TARGET (the
    largest margin tried when none is)."""
    for m in per_margin:
        if m["bler_" + key] <= EVAL_BLER_TARGET:
            return m
    return per_margin[-1]


def evaluate(ctx, net, snrs_db, seed=0, cells=48, max_iterations=6, step_db=EVAL_MARGIN_STEP_DB,
             max_margin_db=EVAL_MARGIN_MAX_DB, verbose=True, min_qm=0):
    """Per SNR, link-adaptation margins 0, step_db, ... until both estimators reach BLER <= 10 % (or
    max_margin_db): BLER (TB CRC and payload against the transmitted bits) of the slot plan with the
    plain and with the learned estimator on the same slots, and the decoded Mbit/s per cell. Each
    estimator then gets its own margin, the smallest with BLER at most 10 % (outer-loop link
    adaptation), and its goodput there; EVM and data-symbol channel NMSE of both at the plain
    estimator's margin."""
    rows = []
    for k, snr in enumerate(snrs_db):
        per_margin, m = [], 0.0
        while True:
            slots = eval_slots(snr, seed + k, cells, la_margin_db=m)
            e_p, b_p = run_plan(ctx, slots, None, max_iterations)
            e_l, b_l = run_plan(ctx, slots, net, max_iterations, min_qm)
            qm = np.array([ue.modulation_order for sl in slots for ue in sl.ues])
            by_qm = {int(q): dict(ues=int((qm == q).sum()), plain=float(np.mean(np.array(e_p)[qm == q])),
                                  learned=float(np.mean(np.array(e_l)[qm == q]))) for q in np.unique(qm)}
            per_margin.append(dict(margin_db=float(m), ues=len(e_p), bler_plain=float(np.mean(e_p)),
                                   bler_learned=float(np.mean(e_l)), bler_by_qm=by_qm,
                                   mbps_plain=b_p / (cells * SLOT_S) / 1e6, mbps_learned=b_l / (cells * SLOT_S) / 1e6))
            done = (any(p["bler_plain"] <= EVAL_BLER_TARGET for p in per_margin) and
                    any(p["bler_learned"] <= EVAL_BLER_TARGET for p in per_margin))
            if done or m + step_db > max_margin_db + 1e-9:
                break
            m += step_db
        lp, ll = la_point(per_margin, "plain"), la_point(per_margin, "learned")
        q = estimate_quality(ctx, eval_slots(snr, seed + k, cells, la_margin_db=lp["margin_db"]), net,
                             max_iterations)
        row = dict(snr_db=float(snr), ues=lp["ues"], margin_plain=lp["margin_db"], margin_learned=ll["margin_db"],
                   bler_plain=lp["bler_plain"], bler_learned_same_mcs=lp["bler_learned"],
                   bler_learned=ll["bler_learned"], mbps_plain=lp["mbps_plain"], mbps_learned=ll["mbps_learned"],
                   evm_plain=q["plain"]["evm"], evm_learned=q["learned"]["evm"], nmse_plain=q["plain"]["nmse"],
                   nmse_learned=q["learned"]["nmse"], per_margin=per_margin)
        rows.append(row)
        if verbose:
            print(("SNR {snr_db:4.1f} dB  UEs {ues:3d}  plain: margin {margin_plain:.0f} BLER {bler_plain:.3f} "
                   "{mbps_plain:7.1f} Mbit/s  learned: same-MCS BLER {bler_learned_same_mcs:.3f}, margin "
                   "{margin_learned:.0f} BLER {bler_learned:.3f} {mbps_learned:7.1f} Mbit/s  EVM {evm_plain:.4f}/"
                   "{evm_learned:.4f}  NMSE {nmse_plain:.5f}/{nmse_learned:.5f}").format(**row), flush=True)
    return rows


def main(argv=None):
    """python -m pusch_b200.learned train|evaluate ... (on a B200)."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m pusch_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="train on the GPU and save the parameters")
    t.add_argument("--steps", type=int, default=13500)
    t.add_argument("--rows", type=int, default=96_000, help="network rows (subcarriers x ports x layers) per step")
    t.add_argument("--seed", type=int, default=0)
    t.add_argument("--lr", type=float, default=1e-3)
    t.add_argument("--time-budget", type=float, default=None, help="stop after this many seconds")
    t.add_argument("--out", default=WEIGHTS)
    t.add_argument("--init", default=None, help="start from the parameters in this file (default: fresh)")
    e = sub.add_parser("evaluate", help="BLER / EVM / NMSE of the plain and learned estimators per SNR")
    e.add_argument("--weights", default=WEIGHTS)
    e.add_argument("--snrs", default="0:30:2", help="first:last:step in dB")
    e.add_argument("--cells", type=int, default=48, help="cells per SNR point and margin (about 10 UEs each)")
    e.add_argument("--seed", type=int, default=100)
    e.add_argument("--json", default=None)
    e.add_argument("--min-qm", type=int, default=0, help="refine only UEs of this modulation order and above")
    tm = sub.add_parser("time", help="time pg_le_refine_device on a batch of the training source")
    tm.add_argument("--rows", type=int, default=270_000)
    tm.add_argument("--reps", type=int, default=50)
    a = ap.parse_args(argv)
    ctx = _native.Context(0, 1024)
    if a.cmd == "time":
        import torch
        src = DmrsTrainingSource(5)
        descs, grid, _, est_size, _ = src.batch(a.rows)
        n = len(descs)
        est = torch.empty(2 * est_size, dtype=torch.float32, device="cuda")
        ls = torch.empty_like(est)
        pr = torch.empty((4 * n, 5), dtype=torch.float32, device="cuda")
        ctx.check(ctx.lib.pg_pusch_estimate_ls_device(ctx.handle, ctypes.addressof(descs), n, grid.data_ptr(),
                                                      est.data_ptr(), ls.data_ptr(), pr.data_ptr(), None))
        rows = int(ctx.lib.pg_le_rows(ctypes.addressof(descs), n))
        net = LearnedEstimator(ctx, max_rows=rows, params=load_params())
        for _ in range(3):
            net.refine(descs, ls.data_ptr(), est.data_ptr(), pr.data_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(a.reps):
            net.refine(descs, ls.data_ptr(), est.data_ptr(), pr.data_ptr())
        e1.record()
        torch.cuda.synchronize()
        net.status()
        ms = e0.elapsed_time(e1) / a.reps
        flops = rows * 2 * TAPS * sum(ci * co for ci, co in LAYERS)
        print(f"rows {rows} refine {ms:.4f} ms {flops / (ms * 1e-3) / 1e12:.1f} TFLOP/s", flush=True)
        net.close()
    elif a.cmd == "train":
        t0 = time.time()
        init = load_params(a.init) if a.init else None
        if a.init and init is None:
            raise SystemExit(f"no parameters at {a.init}")
        net, hist = train(ctx, steps=a.steps, rows_per_step=a.rows, seed=a.seed, lr=a.lr, time_budget_s=a.time_budget,
                          params=init)
        ues_seen = hist[-1][0] * a.rows / (4 * 1.5 * 12 * 92)
        net.save(a.out, history=np.array(hist), steps=hist[-1][0], rows_per_step=a.rows, seed=a.seed,
                 train_seconds=time.time() - t0)
        print(f"saved {a.out}: {hist[-1][0]} steps, about {ues_seen:.0f} UE allocations, "
              f"{time.time() - t0:.1f} s", flush=True)
        net.close()
    else:
        lo, hi, st = (float(v) for v in a.snrs.split(":"))
        snrs = list(np.arange(lo, hi + 1e-9, st))
        params = load_params(a.weights)
        if params is None:
            raise SystemExit(f"no parameters at {a.weights}")
        # A cell holds at most 273 PRB x 4 ports x 2 layers of subcarrier rows, plus the gaps of
        # up to 16 UEs x 8 allocations.
        net = LearnedEstimator(ctx, max_rows=a.cells * (4 * 2 * 12 * 273 + 16 * 8 * 2), params=params)
        rows = evaluate(ctx, net, snrs, seed=a.seed, cells=a.cells, min_qm=a.min_qm)
        if a.json:
            with open(a.json, "w") as f:
                json.dump(rows, f, indent=1)
        net.close()
    ctx.close()


if __name__ == "__main__":
    main()
