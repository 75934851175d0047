"""Benchmark of the B200 TFHE programmable-bootstrapping engine.

Workload: the batched PBS + key-switch throughput case at the 2048
parameter set (uint32 torus, n=742, N=2048, gadget 2^15 x 2, key switch
2^4 x 5, collapse 2), 16384 ciphertexts per step (default), uniform Z_8
messages with a padding bit, each ciphertext with its own LUT drawn from 8
fixed random tables f: Z_8 -> Z_8.  One step = key switch + blind rotation
+ rotation + sample extraction of the whole batch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--batch B]
  python bench.py --impl reference ...   (the CPU statement of the path)

Prints ONE JSON line on rank 0.  ``value`` is device-resident throughput;
``e2e`` is the same metric through tfhe_pbs with host buffers and the
host<->device copies inside the timed region.  Multi-GPU runs are
independent replicas (every PBS is independent; no collective is needed).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "blind-spiking-lstm_b200"))

METRIC = "PBS/s (key switch + blind rotation + many-LUT extraction) at 0 decrypt errors"
UNIT = "PBS/s"
T_MSG = 16           # Z_8 messages with a padding bit: phase m q / 16
T_OUT = 8            # table outputs in Z_8 at scale q / 8 (final outputs, no padding bit)
N_TABLES = 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--params", choices=["cfg2", "cfg1"], default="cfg2",
                    help="engine arm and sweep: the 2048 set (default) or the 1024 set (n=630, gadget 2^7 x 3, c=3)")
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-sample", type=int, default=96, help="ciphertexts in the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-per-core", type=int, default=8,
                    help="ciphertexts per host core in each step of the reference arm")
    ap.add_argument("--no-lstm", action="store_true",
                    help="leave the encrypted Spike-LSTM keys out of the default (PBS) line")
    ap.add_argument("--lstm", action="store_true",
                    help="one encrypted Spike-LSTM layer + head: sequences/s (one GPU)")
    ap.add_argument("--seq-len", type=int, default=32)
    ap.add_argument("--seqs", type=int, default=16)
    ap.add_argument("--hidden", type=int, default=None, help="hidden units (default 128 with --lstm, 256 with --serve)")
    ap.add_argument("--layers", type=int, default=None, help="layers (default 1 with --lstm, 2 with --serve)")
    ap.add_argument("--graph", action="store_true", help="--lstm: replay each timestep from a CUDA graph")
    ap.add_argument("--direct", action="store_true",
                    help="--serve: launch every tick's kernels directly (no CUDA-graph replay of ticks)")
    ap.add_argument("--torus", type=int, choices=[32, 64], default=32,
                    help="--lstm / --serve: the 2^32 torus (config-1 bootstrapping) or the reference's own 2^64")
    ap.add_argument("--serve", action="store_true",
                    help="continuous-batching server with Poisson arrivals: p50/p99 latency and sequences/s")
    ap.add_argument("--rate", type=float, default=2.0, help="requests per second (--serve)")
    ap.add_argument("--requests", type=int, default=48, help="requests per serving run (--serve)")
    ap.add_argument("--max-slots", type=int, default=64)
    ap.add_argument("--clocks-log", default=None,
                    help="file for the nvidia-smi clock samples of the timed region (default: a temporary file)")
    ap.add_argument("--sweep", default=None,
                    help="comma-separated batch sizes: print one line per batch comparing the plain launch with "
                         "the persistent, autotuned, CUDA-graph launch (one GPU)")
    return ap.parse_args()


def flops_per_pbs(p):
    """Algorithmic blind-rotation work per PBS: per group, (2L + 2) H-point
    transforms at 5 H log2 H flops and the pointwise contraction at
    8 H (2 * 2L * M + 2 * 2L) flops (H = N/2), times G groups."""
    H = p.N // 2
    per_group = (2 * p.l_bs + 2) * 5 * H * math.log2(H) + 8 * H * (2 * 2 * p.l_bs * p.M + 2 * 2 * p.l_bs)
    return per_group * p.G


def workload_name(p, batch):
    return (f"PBS+KS n={p.n} N={p.N} gadget 2^{p.log2_beta_bs}x{p.l_bs} KS 2^{p.log2_beta_ks}x{p.l_ks} "
            f"collapse {p.collapse}, batch {batch}, per-ciphertext LUT from {N_TABLES} random Z_8 tables")


# ---------------------------------------------------------------- inputs
def make_inputs(p, batch, seed):
    import numpy as np
    from tfhe_b200 import client
    keys = client.keygen(p, seed)
    rng = np.random.default_rng(seed + 1)
    msgs = rng.integers(0, T_MSG // 2, size=batch)
    a, b = client.encrypt(keys, msgs, T_MSG, rng)
    tables = rng.integers(0, T_MSG // 2, size=(N_TABLES, T_MSG // 2))
    which = rng.integers(0, N_TABLES, size=batch)
    bodies = np.stack([client.table_lut(p.N, tables[i], T_OUT) for i in range(N_TABLES)])
    lut = np.zeros((batch, 2, p.N), dtype=np.uint32)
    lut[:, 1] = bodies[which]
    expect = tables[which, msgs]
    return keys, msgs, a, b, lut, expect


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, path=None):
        self.gpu = gpu_index
        self.proc = None
        # the samples go to the caller's file (--clocks-log) or a temporary one
        self.path = path or os.path.join(tempfile.gettempdir(), f"tfhe_clocks_{os.getpid()}_{gpu_index}.csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        load = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- engine arm
def run_engine(args, rank, world, local_rank, dist):
    import numpy as np
    import torch
    from tfhe_b200 import client
    from tfhe_b200.engine import Keys, launch_count, probe_fp64_peak
    from tfhe_b200.params import CONFIG1, CONFIG2

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    p = CONFIG1 if args.params == "cfg1" else CONFIG2
    B = args.batch
    keys, msgs, a, b, lut, expect = make_inputs(p, B, args.seed + rank)
    eng = Keys.create(p, keys.bsk, keys.ksk_a, keys.ksk_b)
    i32 = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.int32))
    a_h, b_h, lut_h = i32(a).pin_memory(), i32(b).pin_memory(), i32(lut).pin_memory()
    a_d, b_d, lut_d = a_h.to(dev), b_h.to(dev), lut_h.to(dev)
    ka = torch.empty((B, p.n), dtype=torch.int32, device=dev)
    kb = torch.empty((B,), dtype=torch.int32, device=dev)
    oa = torch.empty((B, 1, p.N), dtype=torch.int32, device=dev)
    ob = torch.empty((B, 1), dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream()

    def barrier():
        if dist is not None:
            dist.barrier()

    def step_device(ev=None):
        if ev is not None:
            ev[0].record(stream)
        eng.keyswitch(a_d, b_d, ka, kb)
        if ev is not None:
            ev[1].record(stream)
        eng.cuboot_merge(ka, kb, lut_d, 1, oa, ob)
        if ev is not None:
            ev[2].record(stream)

    for _ in range(args.warmup):
        step_device()
    torch.cuda.synchronize()
    peak_fp64 = probe_fp64_peak()

    clocks = ClockSampler(local_rank, args.clocks_log)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    n_launch0 = launch_count()
    t0.record(stream)
    for s in range(args.steps):
        step_device(evs[s])
    t1.record(stream)
    gpu_launches = launch_count() - n_launch0
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    dev_ms = t0.elapsed_time(t1)
    ks_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    br_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)

    # decryption check of the device outputs
    out_a = oa.cpu().numpy().view(np.uint32)[:, 0]
    out_b = ob.cpu().numpy().view(np.uint32)[:, 0]
    dec = client.decrypt(out_a, out_b, keys.sk_glwe, T_OUT)
    errors = int(np.sum(dec != expect))
    noise = client.phase(out_a, out_b, keys.sk_glwe) - expect.astype(np.int64) * (2 ** 32 // T_OUT)
    noise = ((noise + 2 ** 31) % 2 ** 32) - 2 ** 31
    noise_log2_std = float(np.log2(np.std(noise.astype(np.float64))))

    # end to end through tfhe_pbs_host with host buffers
    oa_h = torch.empty((B, 1, p.N), dtype=torch.int32).pin_memory()
    ob_h = torch.empty((B, 1), dtype=torch.int32).pin_memory()
    def step_e2e():
        # tfhe_pbs_host: host buffers in and out, the uploads / downloads of
        # each chunk overlapped with the compute of its neighbours
        eng.pbs_host(a_h, b_h, lut_h, 1, oa_h, ob_h)

    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    torch.cuda.synchronize()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step_e2e()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)
    e2e_same = bool(torch.equal(oa_h, oa.cpu()) and torch.equal(ob_h, ob.cpu()))

    # max over ranks
    times = torch.tensor([dev_ms, e2e_ms, float(errors), 0.0 if e2e_same else 1.0], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(times, op=dist.ReduceOp.MAX)
    dev_ms, e2e_ms, errors_max, e2e_diff = times.tolist()
    eng.close()
    if rank != 0:
        return None
    lstm = None
    if world == 1 and not args.no_lstm:
        torch.cuda.empty_cache()
        lstm = lstm_summary(args, dev, steps=1, warmup=1, torus_bits=64)
        lstm_q32 = lstm_summary(args, dev, torus_bits=32)
        torch.cuda.empty_cache()
        serving = serving_summary(args)

    total = B * args.steps * world
    value = total / (dev_ms * 1e-3)
    e2e_value = total / (e2e_ms * 1e-3)
    fl = flops_per_pbs(p)
    achieved_tf = B * fl / (br_ms * 1e-3) / 1e12
    traffic = read_traffic(B) if args.params == "cfg2" else None   # the committed capture is of the 2048 set
    line = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dev_ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(p, B), "params": p.name, "batch_per_gpu": B, "n_lut": 1,
                   "parallelism": f"replicas{world}" if world > 1 else "single",
                   "l2": f"inputs larger than L2: {(a_h.numel() + b_h.numel() + lut_h.numel()) * 4 / 1e6:.0f} MB of "
                         f"ciphertexts and LUTs per step, {p.bsk_bytes_fp64() / 1e6:.0f} MB key"},
        "e2e": {"value": round(e2e_value, 1), "unit": UNIT,
                "h2d_bytes_per_step": int(a_h.numel() * 4 + b_h.numel() * 4 + lut_h.numel() * 4),
                "d2h_bytes_per_step": int(oa_h.numel() * 4 + ob_h.numel() * 4),
                "outputs_equal_device_arm": not bool(e2e_diff)},
        "roofline": {"bound": "fp64", "achieved": round(achieved_tf, 3), "peak": round(peak_fp64, 3),
                     "unit": "TFLOP/s", "frac": round(achieved_tf / peak_fp64, 4), "traffic": traffic,
                     "kernel": f"br_fp64_kernel<{p.N.bit_length() - 1},{p.l_bs}> (blind rotation + extraction)",
                     "flops_per_pbs": int(fl), "launch_ms": round(br_ms, 3),
                     "peak_source": "FP64 FMA probe (tfhe_probe_fp64_fma) on this GPU; MEASURED_PEAKS.json "
                                    "holds no FP64 figure",
                     "key_bytes_per_launch": p.bsk_bytes_fp64(),
                     "key_stream_gbs": round(p.bsk_bytes_fp64() / (br_ms * 1e-3) / 1e9, 1),
                     "hbm_view": hbm_view(traffic, br_ms)},
        "kernels_ms": {"keyswitch": round(ks_ms, 3), "blind_rotate_extract": round(br_ms, 3)},
        "decrypt_errors": int(errors_max), "decrypt_checked": B * world,
        "output_noise_log2_std": round(noise_log2_std, 2),
        "gpu_launches": gpu_launches,
        "clocks": clk,
    }
    if lstm is not None:
        line["lstm"] = lstm
        line["lstm_q32"] = lstm_q32
        line["serving"] = serving
    return line


def serving_summary(args):
    """Config 5 as extra keys of the default line: the serving run of
    --serve (Poisson arrivals at 2 requests/s, 24 requests of U[8, 64]
    Zipf(1.1) tokens, 2 layers of hidden 256 on the 2^32 torus, continuous
    batching), reduced to its latency percentiles and throughput."""
    import argparse
    sargs = argparse.Namespace(**vars(args))
    sargs.rate, sargs.requests, sargs.torus, sargs.hidden, sargs.layers = 2.0, 24, 32, None, None
    sargs.warmup = 1
    out = run_serve(sargs)
    return {"workload": "Spike-LSTM serving (config 5): Poisson 2 req/s, 24 requests of U[8,64] tokens, "
                        f"{out['config']['layers']} layers x hidden {out['config']['hidden']}, "
                        f"PBS {out['config']['pbs']}, {out['config']['torus']}",
            "p50_s": out["latency"]["p50_s"], "p99_s": out["latency"]["p99_s"],
            "seq_per_s": out["value"], "tokens_per_s": out["tokens_per_s"], "mean_batch": out["mean_batch"],
            "one_at_a_time_seq_per_s": out["one_at_a_time"]["seq_per_s"],
            "results_equal_to_one_at_a_time": out["one_at_a_time"]["results_equal_to_mix"]}


def lstm_summary(args, dev, steps=2, warmup=1, torus_bits=64):
    """The one-layer encrypted Spike-LSTM workload (16 sequences of 32
    Zipf(1.1) tokens over 8192, embedding 64, hidden 128, 4 packed LUTs,
    weights in [-7, 7], head) timed as extra keys of the PBS line: seq/s on
    device-resident inputs, end to end with the inputs copied from pinned
    host memory and the logits copied back inside the timed region, and the
    plain FP64 per-gate form (one bootstrap launch per gate and sequence,
    one ciphertext per CTA, no persistence or key prefetch, key switch on
    CUDA cores) on the same model and inputs.
    torus_bits 64: the reference's own modulus and bootstrapping parameters
    (q = 2^64, N = 2048, n = 702, gadget 2^13 x 2, collapse 3); 32: the
    config-1 parameters on q = 2^32."""
    import numpy as np
    import torch
    from tfhe_b200 import spike_model as SM

    cfg = SM.config_q64() if torus_bits == 64 else SM.SpikeModelConfig()
    model = SM.build_model(cfg, args.seed)
    dm = SM.to_device(model, dev)
    rng = np.random.default_rng(args.seed + 5)
    S, T = 16, 32
    tokens = SM.sample_tokens(rng, S, T, cfg.vocab, cfg.zipf)
    xs_h = SM.encrypted_words(model, SM.encrypt_tokens(model, tokens, rng)).pin_memory()
    xs_d = xs_h.to(dev)
    stream = torch.cuda.current_stream()
    pbs = dm.keys.pbs
    tunable = hasattr(pbs, "set_tuning")

    def forward(xs, per_gate=False):
        H, _ = SM.run_layers(dm, xs, per_gate=per_gate)
        return dm.head(H)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps, out

    dev_ms, (la, lb) = timed(lambda: forward(xs_d))
    la_h = torch.empty(la.shape, dtype=la.dtype).pin_memory()
    lb_h = torch.empty(lb.shape, dtype=lb.dtype).pin_memory()
    xs_e = torch.empty_like(xs_d)

    def e2e():
        xs_e.copy_(xs_h, non_blocking=True)
        a, b = forward(xs_e)
        la_h.copy_(a, non_blocking=True)
        lb_h.copy_(b, non_blocking=True)
        return a, b

    e2e_ms, _ = timed(e2e)
    if tunable:
        pbs.set_tuning(1, 0, 0, 0, 0)
    gate_ms, (ga, gb) = timed(lambda: forward(xs_d, per_gate=True))
    if tunable:
        pbs.set_tuning()
    same = bool(torch.equal(ga, la) and torch.equal(gb, lb))
    logits = SM.decrypt_logits(model, la_h, lb_h)
    plain, _ = SM.plain_forward(model, tokens)
    return {"workload": f"one-layer encrypted Spike-LSTM: {S} sequences x {T} Zipf(1.1) tokens over {cfg.vocab}, "
                        f"embedding {cfg.emb_dim}, hidden {cfg.hidden}, {cfg.n_lut} packed LUTs, weights [-7, 7], "
                        f"head; PBS {cfg.pbs.name}; torus q = 2^{torus_bits}",
            "seq_per_s": round(S / dev_ms * 1e3, 3), "ms_per_batch": round(dev_ms, 2),
            "e2e_seq_per_s": round(S / e2e_ms * 1e3, 3),
            "e2e_bytes": {"h2d": int(xs_h.numel() * 4), "d2h": int((la_h.numel() + lb_h.numel()) * 4)},
            "plain_fp64_per_gate_seq_per_s": round(S / gate_ms * 1e3, 3),
            "speedup_vs_plain_per_gate": round(gate_ms / dev_ms, 3),
            "outputs_equal_per_gate": same,
            "logit_sign_agreement_vs_plaintext": float(np.mean(np.sign(logits) == np.sign(plain))),
            "steps": steps, "warmup": warmup}


def run_lstm(args):
    """Encrypted Spike-LSTM: token ids Zipf(1.1) over 8192, int embeddings
    of dim 64 encrypted per timestep, hidden 128 (4 packed LUTs per
    bootstrap), 3 gate linears with weights in [-7, 7], head linear + ReLU
    bootstrap + packing + linear; `seqs` sequences of `seq_len` tokens per
    step.  value: sequences/s with encrypted inputs resident on the GPU;
    e2e: the same with the host -> device copy of every step's inputs and
    the device -> host copy of the logits inside the timed region."""
    import numpy as np
    import torch
    from tfhe_b200 import spike_model as SM
    from tfhe_b200.engine import launch_count

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    hidden = args.hidden or 128
    layers = args.layers or 1
    cfg = (SM.config_q64(hidden=hidden, layers=layers) if args.torus == 64
           else SM.SpikeModelConfig(hidden=hidden, layers=layers))
    model = SM.build_model(cfg, args.seed)
    dm = SM.to_device(model, dev)
    rng = np.random.default_rng(args.seed + 5)
    tokens = SM.sample_tokens(rng, args.seqs, args.seq_len, cfg.vocab, cfg.zipf)
    xs_h = SM.encrypted_words(model, SM.encrypt_tokens(model, tokens, rng)).pin_memory()
    xs_d = xs_h.to(dev)
    stream = torch.cuda.current_stream()

    graphs = None
    if args.graph:
        from tfhe_b200.lstm import StepGraph
        if cfg.layers != 1:
            raise SystemExit("--graph supports one layer")
        graphs = StepGraph(dm.layers[0], args.seqs)

    def forward(xs):
        if graphs is not None:
            H, _ = graphs.run(xs)
        else:
            H, _ = SM.run_layers(dm, xs)
        return dm.head(H)

    for _ in range(args.warmup):
        forward(xs_d)
    torch.cuda.synchronize()
    clocks = ClockSampler(0, args.clocks_log)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_launch0 = launch_count()
    e0.record(stream)
    for _ in range(args.steps):
        la, lb = forward(xs_d)
    e1.record(stream)
    gpu_launches = launch_count() - n_launch0
    torch.cuda.synchronize()
    dev_ms = e0.elapsed_time(e1) / args.steps
    clk = clocks.stop()

    la_h = torch.empty(la.shape, dtype=la.dtype).pin_memory()
    lb_h = torch.empty(lb.shape, dtype=lb.dtype).pin_memory()
    xs_e = torch.empty_like(xs_d)
    e0.record(stream)
    for _ in range(args.steps):
        xs_e.copy_(xs_h, non_blocking=True)
        a, b = forward(xs_e)
        la_h.copy_(a, non_blocking=True)
        lb_h.copy_(b, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps

    logits = SM.decrypt_logits(model, la_h, lb_h)
    plain, _ = SM.plain_forward(model, tokens)
    pbs_per_seq = args.seq_len * cfg.layers * 3 * (cfg.hidden // cfg.n_lut) + cfg.hidden
    return {"metric": "encrypted Spike-LSTM sequences/s (layer + head)", "value": round(args.seqs / dev_ms * 1e3, 3),
            "unit": "seq/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dev_ms, 2), "higher_is_better": True,
            "dtype": f"u{cfg.torus_bits} torus, f64 FFT",
            "data": "synthetic: Zipf(1.1) tokens over 8192, random int weights / embeddings / thresholds",
            "config": {"workload": "Spike-LSTM", "seqs": args.seqs, "seq_len": args.seq_len, "emb_dim": cfg.emb_dim,
                       "timestep": "CUDA graph" if args.graph else "direct launches",
                       "hidden": cfg.hidden, "layers": cfg.layers, "n_lut": cfg.n_lut, "pbs": cfg.pbs.name,
                       "weights": "[-7, 7]"},
            "e2e": {"value": round(args.seqs / e2e_ms * 1e3, 3), "unit": "seq/s",
                    "h2d_bytes_per_step": int(xs_h.numel() * 4), "d2h_bytes_per_step": int((la.numel() + lb.numel()) * 4)},
            "pbs_per_sequence": pbs_per_seq, "pbs_per_s": round(pbs_per_seq * args.seqs / dev_ms * 1e3, 1),
            "gpu_launches": gpu_launches,
            "decrypted_logits": [round(float(v), 2) for v in logits[:8]],
            "plain_logits": [round(float(v), 2) for v in plain[:8]],
            "logit_sign_agreement": float(np.mean(np.sign(logits) == np.sign(plain))),
            "logit_mean_abs_diff": round(float(np.mean(np.abs(logits - plain))), 3),
            "clocks": clk}


def run_serve(args):
    """Serving: Poisson arrivals at --rate requests/s; each request an
    encrypted sequence of U[8, 64] Zipf(1.1) tokens; 2-layer Spike-LSTM with
    hidden 256 (layers and hidden from the flags when given), per-request
    encrypted state kept on the GPU, continuous batching (every live
    request's current timestep in one batched step; ticks replayed from CUDA
    graphs per combination of request counts, or launched directly with
    --direct).  Reports p50/p99 latency and sequences/s, next to the same
    requests served one at a time (one slot: no batching across requests)."""
    import numpy as np
    import torch
    from tfhe_b200 import spike_model as SM
    from tfhe_b200.serving import DeviceStepModel, Request, SpikeLstmServer, latency_summary, run_arrivals, \
        slots_for_memory

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    hidden = args.hidden or 256
    layers = args.layers or 2
    cfg = (SM.config_q64(hidden=hidden, layers=layers) if args.torus == 64
           else SM.SpikeModelConfig(hidden=hidden, layers=layers))
    model = SM.build_model(cfg, args.seed)
    dm = SM.to_device(model, dev)
    sm = DeviceStepModel(dm, graphs=False if getattr(args, "direct", False) else None)
    rng = np.random.default_rng(args.seed + 9)
    t_max = 64
    free, _ = torch.cuda.mem_get_info()
    slots = slots_for_memory(sm, t_max, free, 16 << 30, args.max_slots)

    def make_requests(n, rate):
        gaps = rng.exponential(1.0 / rate, size=n)
        arr = np.cumsum(gaps) - gaps[0]
        out = []
        for i in range(n):
            T = int(rng.integers(8, 65))
            tok = SM.sample_tokens(rng, 1, T, cfg.vocab, cfg.zipf)
            xs = SM.encrypted_words(model, SM.encrypt_tokens(model, tok, rng))[:, 0].contiguous().pin_memory()
            out.append(Request(i, xs, arrival=float(arr[i])))
        return out

    # warm-up: the ticks of up to four requests per layer captured as graphs
    # ahead of the timed run, then two short requests through a server
    sm.warm_graphs(4)
    warm = SpikeLstmServer(sm, 2, t_max, dev)
    for r in make_requests(2, 100.0):
        r.xs = r.xs[:2].contiguous()
        warm.submit(r)
    for _ in range(max(1, args.warmup)):
        warm.tick()
    torch.cuda.synchronize()

    reqs = make_requests(args.requests, args.rate)
    clocks = ClockSampler(0, args.clocks_log)
    clocks.start()
    srv = SpikeLstmServer(sm, slots, t_max, dev)
    done = run_arrivals(srv, reqs)
    torch.cuda.synchronize()
    clk = clocks.stop()
    span = max(r.done for r in done) - min(r.arrival for r in done)
    lat = latency_summary(done)

    # the same first few requests one at a time, back to back
    k = min(6, len(reqs))
    solo = SpikeLstmServer(sm, 1, t_max, dev)
    import time as _t
    t0 = _t.perf_counter()
    solo_reqs = [Request(r.rid, r.xs, arrival=0.0) for r in reqs[:k]]
    for r in solo_reqs:
        r.arrival = _t.perf_counter()
        solo.submit(r)
        while not solo.idle():
            solo.tick()
    solo_span = _t.perf_counter() - t0
    same = all(torch.equal(a.logits[0], b.logits[0]) and torch.equal(a.logits[1], b.logits[1])
               for a, b in zip(solo_reqs, reqs[:k]))
    tokens = sum(r.length for r in done)
    return {"metric": "encrypted Spike-LSTM serving: p50/p99 latency and sequences/s", "value": round(len(done) / span, 3),
            "unit": "seq/s", "n_gpus": 1, "higher_is_better": True, "dtype": "u32 torus, f64 FFT",
            "data": "synthetic: Poisson arrivals, U[8,64] Zipf(1.1) tokens, random int weights",
            "config": {"workload": "Spike-LSTM serving", "rate_req_per_s": args.rate, "requests": len(done),
                       "layers": cfg.layers, "hidden": cfg.hidden, "emb_dim": cfg.emb_dim, "n_lut": cfg.n_lut,
                       "slots": slots, "pbs": cfg.pbs.name, "torus": f"q = 2^{cfg.torus_bits}",
                       "ticks": "direct launches" if sm.graphs is None else "CUDA-graph replay"},
            "latency": {k2: (round(v, 3) if isinstance(v, float) else v) for k2, v in lat.items()},
            "tokens_per_s": round(tokens / span, 2), "ticks": srv.ticks,
            "mean_batch": round(float(np.mean(srv.batch_sizes)), 2), "max_batch": int(max(srv.batch_sizes)),
            "one_at_a_time": {"requests": k, "seq_per_s": round(k / solo_span, 3),
                              "results_equal_to_mix": bool(same)},
            "clocks": clk}


def run_sweep(args, batches):
    """Batch sweep at the 2048 parameter set: for every batch size, three
    arms on the same inputs: the plain FP64 per-gate form (one ciphertext per
    CTA, grid = batch, no persistence or key prefetch, key switch on CUDA
    cores), the automatic shape on a non-persistent grid (direct calls), and
    the persistent, autotuned launch replayed from a CUDA graph.  Every arm
    times key switch + blind rotation + extraction on device-resident inputs
    with CUDA events and decrypts every output."""
    import numpy as np
    import torch
    from tfhe_b200 import client
    from tfhe_b200.autotune import autotune
    from tfhe_b200.engine import Keys, PBSGraph
    from tfhe_b200.params import CONFIG1, CONFIG2

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    p = CONFIG1 if args.params == "cfg1" else CONFIG2
    bmax = max(batches)
    keys, msgs, a, b, lut, expect = make_inputs(p, bmax, args.seed)
    eng = Keys.create(p, keys.bsk, keys.ksk_a, keys.ksk_b)
    i32 = lambda x: torch.from_numpy(np.ascontiguousarray(x).view(np.int32)).to(dev)
    a_d, b_d, lut_d = i32(a), i32(b), i32(lut)
    stream = torch.cuda.current_stream()
    out = []
    for B in batches:
        steps = max(args.steps, min(200, 65536 // max(B, 1)))
        ka = torch.empty((B, p.n), dtype=torch.int32, device=dev)
        kb = torch.empty((B,), dtype=torch.int32, device=dev)
        oa = torch.empty((B, 1, p.N), dtype=torch.int32, device=dev)
        ob = torch.empty((B, 1), dtype=torch.int32, device=dev)

        def timed(fn):
            for _ in range(args.warmup):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / steps

        def errors(out_a, out_b):
            dec = client.decrypt(out_a.cpu().numpy().view(np.uint32)[:, 0], out_b.cpu().numpy().view(np.uint32)[:, 0],
                                 keys.sk_glwe, T_OUT)
            return int(np.sum(dec != expect[:B]))

        def direct():
            eng.keyswitch(a_d[:B], b_d[:B], ka, kb)
            eng.cuboot_merge(ka, kb, lut_d[:B], 1, oa, ob)

        # the plain FP64 form: one ciphertext per CTA and one CTA per
        # ciphertext (grid = batch, as the reference's mul_bootstrap kernel
        # launches), no persistence, no key prefetch into L2 or L1, key switch
        # on CUDA cores
        eng.set_tuning(1, 0, 0, 0, 0)
        gate_ms = timed(direct)
        gate_err = errors(oa, ob)
        gate_a, gate_b = oa.clone(), ob.clone()
        # the engine's automatic shape on a non-persistent grid
        eng.set_tuning(0, -1, 0)
        plain_ms = timed(direct)
        plain_err = errors(oa, ob)
        plain_shape = eng.launch_shape(B)

        shape, _ = autotune(eng, B, use_cache=False, reps=2)
        graph = PBSGraph(eng, B, n_lut=1, lut_count=B)
        graph.lut.copy_(lut_d[:B])
        graph.a.copy_(a_d[:B])
        graph.b.copy_(b_d[:B])
        tuned_ms = timed(graph.graph.replay)
        tuned_err = errors(graph.out_a, graph.out_b)
        same = bool(torch.equal(graph.out_a, oa) and torch.equal(graph.out_b, ob) and torch.equal(gate_a, oa)
                    and torch.equal(gate_b, ob))
        del graph
        eng.set_tuning()
        out.append({"sweep": f"PBS+KS n={p.n} N={p.N} gadget 2^{p.log2_beta_bs}x{p.l_bs} KS 2^{p.log2_beta_ks}x{p.l_ks} "
                              f"c={p.collapse}", "batch": B, "steps": steps,
                    "plain_fp64_per_gate": {"ms_per_batch": round(gate_ms, 4), "PBS/s": round(B / gate_ms * 1e3, 1),
                                            "decrypt_errors": gate_err, "K": 1, "grid": B, "persistent": 0,
                                            "key_prefetch": "off", "key_switch": "CUDA cores"},
                    "plain": {"ms_per_batch": round(plain_ms, 4), "PBS/s": round(B / plain_ms * 1e3, 1),
                              "decrypt_errors": plain_err, "K": plain_shape[0], "persistent": 0},
                    "persistent_autotuned_graph": {"ms_per_batch": round(tuned_ms, 4),
                                                   "PBS/s": round(B / tuned_ms * 1e3, 1),
                                                   "decrypt_errors": tuned_err,
                                                   "shape": {"K": shape[0], "prefetch": shape[1],
                                                             "persistent": shape[2]}},
                    "outputs_equal": same, "speedup": round(plain_ms / tuned_ms, 3),
                    "speedup_vs_per_gate": round(gate_ms / tuned_ms, 3)})
    eng.close()
    return out


def hbm_view(traffic, launch_ms):
    """The same launch against the HBM roofline: DRAM bytes (ncu-derived,
    scaled to the launch) per launch time over the measured copy bandwidth
    of MEASURED_PEAKS.json, or the pool's earlier copy measurement of
    6.65 TB/s when that file is absent (said in peak_source)."""
    if traffic is None:
        return None
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, source = 6650.0, "fallback 6.65 TB/s (earlier copy measurement; MEASURED_PEAKS.json absent)"
    try:
        peak = float(json.load(open(path))["hbm_gbs"])
        source = "MEASURED_PEAKS.json hbm_gbs (measured copy)"
    except (OSError, ValueError, KeyError, TypeError):
        pass
    gbs = traffic / (launch_ms * 1e-3) / 1e9
    return {"achieved_gbs": round(gbs, 1), "peak_gbs": peak, "frac": round(gbs / peak, 4),
            "peak_source": source}


def read_traffic(batch):
    """DRAM bytes per launch of the blind-rotation kernel from the committed
    ncu summary (bytes per ciphertext of a captured launch), or None."""
    path = os.path.join(ROOT, "profiles", "br_fp64_cfg2_traffic.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_ciphertext"):
            return int(float(line.split("=")[1]) * batch)
    return None


# ---------------------------------------------------------------- CPU statement
def _oracle_worker_init(seed):
    global _W
    import numpy as np
    from oracle import tfhe_oracle as O
    from tfhe_b200 import client
    from tfhe_b200.params import CONFIG2
    p = CONFIG2
    keys = client.keygen(p, seed)
    cen = lambda u: np.asarray(u, dtype=np.uint32).view(np.int32).astype(np.float64)
    _W = dict(p=p, keys=keys, cen=cen, bo=O.bsk_coeff_fourier_ordered(cen(keys.bsk)),
              rot=O.all_rot_possible_fourier(p.N), ksk=(cen(keys.ksk_a), cen(keys.ksk_b)[..., None]))


def _oracle_pbs(chunk):
    """KS + FP64 blind rotation + extraction of the numpy statement of the
    reference (schemas/LWE_jax.py:97-117, schemas/RLWE_jax.py:288-303)."""
    import numpy as np
    from oracle import tfhe_oracle as O
    from tfhe_b200 import client
    w = _W
    p, cen = w["p"], w["cen"]
    a, b, lut = chunk
    t0 = time.perf_counter()
    ca, cb = O.key_switch_LWE(w["ksk"], (cen(a), cen(b)[:, None]),
                              {"beta_ks": 2 ** p.log2_beta_ks, "l_ks": p.l_ks, "q": p.q})
    oa, ob = O.cuboot_merge((ca, cb), [cen(lut[:, 0]), cen(lut[:, 1])], w["bo"], p.q, 2 ** p.log2_beta_bs,
                            p.l_bs, p.N, p.collapse, w["rot"], 1)
    dt = time.perf_counter() - t0
    dec = client.decrypt(client._u32(oa[:, 0]), client._u32(ob[:, 0, 0]), w["keys"].sk_glwe, T_OUT)
    return dt, dec


class CpuStatement:
    """Process pool (spawned before any GPU work) timing the numpy statement
    of the path; every worker derives the same keys from the seed."""

    def __init__(self, seed, workers):
        import multiprocessing as mp
        self.workers = workers
        self.pool = mp.get_context("spawn").Pool(workers, initializer=_oracle_worker_init, initargs=(seed,))

    def run(self, a, b, lut):
        import numpy as np
        w = self.workers
        chunks = [(a[i::w], b[i::w], lut[i::w]) for i in range(w) if len(a[i::w])]
        t0 = time.perf_counter()
        res = self.pool.map(_oracle_pbs, chunks)
        wall = time.perf_counter() - t0
        dec = np.empty(len(a), dtype=np.int64)
        for i, (_, d) in enumerate(res):
            dec[i::w] = d
        return wall, dec

    def close(self):
        self.pool.close()
        self.pool.join()


def cpu_sample(seed, count, workers):
    """PBS/s of the numpy statement on `count` ciphertexts of the workload."""
    import numpy as np
    from tfhe_b200.params import CONFIG2
    keys, msgs, a, b, lut, expect = make_inputs(CONFIG2, count, seed)
    st = CpuStatement(seed, workers)
    try:
        st.run(a[:workers], b[:workers], lut[:workers])          # warm-up
        wall, dec = st.run(a, b, lut)
    finally:
        st.close()
    return count / wall, wall, int(np.sum(dec != expect))


def _set_single_thread():
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"


def run_reference(args, rank, world):
    """The reference arm: the CPU statement of the path timed on the host
    cores with all threads (one process per core), on the engine arm's
    workload; each step is a bounded sample of --ref-per-core ciphertexts per
    core (one batch per process, as the reference's batched path would)."""
    if rank != 0:
        return None
    import numpy as np
    from tfhe_b200.params import CONFIG2
    cores = os.cpu_count() or 1
    per = max(1, args.ref_per_core)
    steps = args.warmup + args.steps
    keys, msgs, a, b, lut, expect = make_inputs(CONFIG2, cores * per * steps, args.seed)
    st = CpuStatement(args.seed, cores)
    walls, errors = [], 0
    try:
        for s in range(steps):
            sl = slice(s * cores * per, (s + 1) * cores * per)
            wall, dec = st.run(a[sl], b[sl], lut[sl])
            if s >= args.warmup:
                walls.append(wall)
                errors += int(np.sum(dec != expect[sl]))
    finally:
        st.close()
    wall = sum(walls)
    value = cores * per * args.steps / wall
    sample = f"{cores * per} ciphertexts per step ({per} per process, {cores} processes) of the batch-{args.batch} workload"
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * wall / args.steps, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(CONFIG2, args.batch), "n_lut": 1},
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": sample + "; numpy statement of the reference JAX path (oracle/)"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "decrypt_errors": errors,
        "note": "the reference's own CUDA kernel needs cuFFTDx and the XLA FFI headers, absent here; "
                "its JAX path needs jax, absent here; the CPU arm is the numpy statement of that path",
    }


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        _set_single_thread()
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return 0

    if args.lstm:
        print(json.dumps(run_lstm(args)), flush=True)
        return 0

    if args.serve:
        print(json.dumps(run_serve(args)), flush=True)
        return 0

    if args.sweep:
        for line in run_sweep(args, [int(x) for x in args.sweep.split(",")]):
            print(json.dumps(line), flush=True)
        return 0

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # bounded CPU sample before any CUDA work (spawned workers)
        _set_single_thread()
        rate, wall, err = cpu_sample(args.seed + 99, args.cpu_sample, 1)
        cpu = {"value": round(rate, 3), "unit": UNIT, "cores": 1, "kind": "port",
               "sample": f"{args.cpu_sample} ciphertexts of the same workload (key switch + FP64 blind rotation "
                         f"+ extraction), numpy statement of the reference JAX path, 1 thread, {wall:.1f} s",
               "decrypt_errors": err}

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    line = run_engine(args, rank, world, local_rank, dist)
    if line is not None:
        line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
