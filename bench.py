"""Benchmark: SCRS erasure-coding hot path on B200.

    python bench.py --gpus N --steps K --warmup W [--impl reference] [--no-extras]

Headline workload (GF(256) Good Cauchy, k=10, m=4, symbol_len=4096): per GPU
and per step, 65536 stripes are encoded and 65536 stripes are batch-decoded
(each from a seeded random choice of 10 of the 14 codeword symbols, so up to
4 data symbols are erased), all in ONE persistent launch replayed from a CUDA
graph, with a device-side plan kernel that builds every stripe's decode
matrix.  Inputs (5.4 GB per GPU) are far larger than the 126 MB L2, so no L2
flush is needed between steps.

`value` is goodput: data bytes (k * symbol_len per encoded or decoded stripe,
the reference's criterion convention) per second over the whole job, with
inputs already in HBM.  `e2e` is the same metric through the C ABI's
host-buffer batch entry point: every step copies the inputs from pinned host
memory and copies the repairs and decoded data back inside the timed region.
`roofline` is the persistent multiply-XOR kernel's algorithmic bytes per launch
(encode (k+m)*L, decode 2*k*L per stripe) over its CUDA-event duration,
against the measured HBM copy bandwidth.  `cpu_baseline` is the CPU
restatement of the reference (oracle/, GFNI payload kernels, all host
threads) on a bounded sample of the same workload.

Multi-GPU: stripes are independent units, so every rank runs its own 65536 +
65536 stripes (weak scaling, no data-path collective); the step time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import gc
import json
import os
import re
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "encode/decode GB/s and HBM-roofline % on 1 B200; batched vs plain; p50/p99 ms"
K, M, L = 10, 4, 4096
STRIPES = 65536
MIXED_STRIPES = 8192  # stripes of the mixed batch; smaller values are for ncu captures
ENVELOPE_CELLS = None  # (k, m) cells of the GF(256) envelope; None: the full 3 x 3 sweep
ENVELOPE_BYTES = 512 << 20  # input bytes per envelope cell
CALL_REPS = None  # per-call extras: calls per mean / percentile (None: 20 / 200); small values for ncu launch lists
SEED = 0x5C250001


def workload() -> str:
    return (f"GF(256) Good Cauchy k={K} m={M} symbol_len={L}: {STRIPES} stripes encoded + {STRIPES} stripes "
            f"batch-decoded from seeded random {K}-of-{K + M} symbol sets, per GPU per step, one persistent "
            "launch (CUDA graph)")


def input_bytes() -> int:
    """Device bytes read by one step: k data rows per encoded stripe, k received rows per decoded stripe."""
    return 2 * STRIPES * K * L


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic_ratio():
    """DRAM bytes per algorithmic byte of the drain kernel, from the committed
    ncu summary (profiles/), or None when no capture has been summarised."""
    f = ROOT / "profiles" / "gf256_mxk_cfg1_ncu.md"
    if not f.exists():
        return None
    m = re.search(r"traffic_per_algorithmic_byte:\s*([0-9.]+)", f.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        self.result = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if not self.proc:
            return
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sms, mx, reasons = [], None, set()
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm, smax, pwr = float(parts[1]), float(parts[2]), float(parts[3])
            except ValueError:
                continue
            mx = smax
            if pwr > 200:  # under load
                sms.append(sm)
                for name, col in (("hw_slowdown", 5), ("hw_thermal_slowdown", 6), ("sw_thermal_slowdown", 7),
                                  ("sw_power_cap", 8)):
                    if parts[col].lower().startswith("active"):
                        reasons.add(name)
        self.result = {"sm_mhz": float(np.median(sms)) if sms else None, "sm_max_mhz": mx,
                       "reasons": sorted(reasons), "samples": len(sms)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=None)
    return world, rank, local


def barrier_max(value: float, world: int) -> float:
    from scrs_b200.shard import max_over_ranks

    return value if world == 1 else max_over_ranks(value)


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


# ---------------------------------------------------------------------------
# workload construction
# ---------------------------------------------------------------------------

def build_cfg1(torch, api, rank):
    """Device-resident cfg1 batch: S encode stripes + S decode stripes."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import OP_DECODE, OP_ENCODE, StripeBatch

    S = STRIPES
    gen = torch.Generator(device="cuda")
    gen.manual_seed(SEED + rank)
    data = torch.randint(0, 256, (S, K * L), dtype=torch.uint8, device="cuda", generator=gen)
    repairs = torch.zeros((S, M * L), dtype=torch.uint8, device="cuda")
    # one encode pass produces the codewords the decode stripes receive from
    b = StripeBatch(api.lib, 2 * S)
    ptr_d, ptr_r = data.data_ptr(), repairs.data_ptr()
    eng = int(Engine.GOOD_CAUCHY)
    idx_enc = np.arange(S, dtype=np.uint64)
    b.set_arrays(np.full(S, OP_ENCODE), np.full(S, eng), np.full(S, K), np.full(S, M), np.full(S, L),
                 ptr_d + idx_enc * (K * L), ptr_r + idx_enc * (M * L))
    b.run()
    torch.cuda.synchronize()
    rng = np.random.default_rng(SEED + 17 + rank)
    # seeded random 10-of-14 received sets, in random arrival order
    keys = rng.random((S, K + M))
    recv = np.argsort(keys, axis=1)[:, :K].astype(np.int64)
    word = torch.cat([data.view(S, K, L), repairs.view(S, M, L)], dim=1)
    received = word[torch.arange(S, device="cuda")[:, None], torch.from_numpy(recv).cuda()].reshape(S, K * L)
    del word
    decoded = torch.zeros((S, K * L), dtype=torch.uint8, device="cuda")
    op = np.concatenate([np.full(S, OP_ENCODE), np.full(S, OP_DECODE)])
    ins = np.concatenate([ptr_d + idx_enc * (K * L), received.data_ptr() + idx_enc * (K * L)])
    outs = np.concatenate([ptr_r + idx_enc * (M * L), decoded.data_ptr() + idx_enc * (K * L)])
    indices = np.zeros((2 * S, K), dtype=np.uint16)
    indices[S:] = recv
    b.set_arrays(op, np.full(2 * S, eng), np.full(2 * S, K), np.full(2 * S, M), np.full(2 * S, L), ins, outs,
                 indices=indices)
    return dict(batch=b, data=data, repairs=repairs, received=received, decoded=decoded, recv=recv)


def verify_cfg1(torch, api, w, oracle_api=None, n_check=8):
    """Decoded data must equal the original data (bit-exact); a sample of repairs
    is compared with the oracle when it is available."""
    ok = bool(torch.equal(w["decoded"], w["data"]))
    if oracle_api is not None and ok:
        from scrs_b200.api import Engine

        p = oracle_api.resolve(Engine.GOOD_CAUCHY, K, M, L)
        enc = oracle_api.batch_encoder(p)
        for s in range(0, STRIPES, max(1, STRIPES // n_check)):
            exp = np.zeros(M * L, np.uint8)
            enc.encode_into(w["data"][s].cpu().numpy(), exp)
            ok &= bool(np.array_equal(exp, w["repairs"][s].cpu().numpy()))
    return ok


def h2d_rate(torch, h_src) -> float:
    """GB/s of one 1 GiB pinned host-to-device copy (median of three),
    timed with CUDA events: the link rate e2e is bound by."""
    n = min(1 << 30, h_src.numel())
    src = h_src.view(-1)[:n]
    dst = torch.empty(n, dtype=torch.uint8, device="cuda")
    ts = []
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        dst.copy_(src, non_blocking=True)
        e.record()
        torch.cuda.synchronize()
        ts.append(s.elapsed_time(e))
    del dst
    return n / (float(np.median(ts)) / 1e3) / 1e9


def bench_config(world) -> dict:
    """The workload's description, identical in both arms' lines."""
    return {"workload": workload(), "engine": "GoodCauchy", "k": K, "m": M, "symbol_len": L,
            "stripes_encode": STRIPES, "stripes_decode": STRIPES, "goodput_bytes_per_step": goodput_bytes(),
            "l2": (f"inputs {input_bytes() / 1e9:.2f} GB per GPU > 126 MB L2, no flush needed"
                   if input_bytes() > 126 << 20 else
                   f"inputs {input_bytes() / 1e6:.1f} MB per GPU fit in the 126 MB L2 (small case)"),
            "parallelism": f"weak x{world}"}


def goodput_bytes():
    return 2 * STRIPES * K * L  # k*L per encoded and per decoded stripe


def algorithmic_bytes():
    return STRIPES * (K + M) * L + STRIPES * 2 * K * L


# ---------------------------------------------------------------------------
# CPU baseline (oracle): bounded sample of the same workload
# ---------------------------------------------------------------------------

def load_oracle():
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
    lib = C.CDLL(str(ROOT / "oracle" / "_build" / "liboracle.so"))
    lib.oracle_baseline_gf256_encode.restype = C.c_double
    lib.oracle_baseline_gf256_encode.argtypes = [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                                 C.c_void_p, C.c_uint64, C.c_int32]
    lib.oracle_baseline_gf256_decode.restype = C.c_double
    lib.oracle_baseline_gf256_decode.argtypes = [C.c_int32, C.c_uint64, C.c_uint64, C.c_uint64, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32]
    lib.oracle_baseline_stripes.restype = C.c_double
    lib.oracle_baseline_stripes.argtypes = [C.c_void_p, C.c_uint64, C.c_int32, C.POINTER(C.c_int32)]
    lib.oracle_baseline_threads.restype = C.c_int32
    lib.oracle_simd_active.restype = C.c_int32
    return lib


def host_cpu() -> dict:
    """Model and logical CPU count of the host the CPU legs run on."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


class CpuSample:
    def __init__(self, lib, count):
        self.lib = lib
        self.count = count
        rng = np.random.default_rng(SEED)
        self.data = rng.integers(0, 256, count * K * L, dtype=np.uint8)
        self.rep = np.zeros(count * M * L, np.uint8)
        self.threads = lib.oracle_baseline_threads()
        lib.oracle_baseline_gf256_encode(1, K, M, L, self.data.ctypes.data, self.rep.ctypes.data, count,
                                         self.threads)
        recv = np.argsort(rng.random((count, K + M)), axis=1)[:, :K]
        word = np.concatenate([self.data.reshape(count, K, L), self.rep.reshape(count, M, L)], axis=1)
        self.received = np.ascontiguousarray(word[np.arange(count)[:, None], recv]).reshape(-1)
        self.indices = np.ascontiguousarray(recv.astype(np.uint16))
        self.out = np.zeros(count * K * L, np.uint8)

    def step(self):
        t1 = self.lib.oracle_baseline_gf256_encode(1, K, M, L, self.data.ctypes.data, self.rep.ctypes.data,
                                                   self.count, self.threads)
        t2 = self.lib.oracle_baseline_gf256_decode(1, K, M, L, self.received.ctypes.data,
                                                   self.indices.ctypes.data, self.out.ctypes.data, self.count,
                                                   self.threads)
        return t1 + t2

    def goodput_bytes(self):
        return 2 * self.count * K * L


def cpu_baseline(target_s=12.0, sample_pairs=8192):
    """The oracle on all host threads over a bounded sample of the workload:
    `sample_pairs` encode + decode stripes, repeated for about target_s."""
    lib = load_oracle()
    samp = CpuSample(lib, min(sample_pairs, STRIPES))
    samp.step()
    times = []
    t_end = time.perf_counter() + target_s
    while time.perf_counter() < t_end or len(times) < 3:
        times.append(samp.step())
    dt = float(np.mean(times))
    ok = np.array_equal(samp.out, samp.data)
    # one thread, as the reference runs one codec per call (a few seconds)
    all_threads = samp.threads
    samp.threads = 1
    one = [samp.step() for _ in range(2)]
    samp.threads = all_threads
    single = samp.goodput_bytes() / float(np.mean(one)) / 1e9
    return {"value": round(samp.goodput_bytes() / dt / 1e9, 3), "unit": "GB/s", "cores": samp.threads,
            "kind": "port", "single_core_GBps": round(single, 3), "cpu": host_cpu(),
            "sample": f"{samp.count} stripes encoded + {samp.count} batch-decoded (k=10 m=4 L=4096) per pass, "
                      f"{len(times)} passes in {sum(times):.1f} s on {samp.threads} threads, "
                      f"GFNI={'on' if lib.oracle_simd_active() else 'off'}, decode {'bit-exact' if ok else 'MISMATCH'}"}


class Cpu:
    """The CPU legs of the extras: the oracle (the CPU restatement of the
    reference's engines, GFNI payload kernels) as a library of host-thread
    baselines and as the Python-bound checker."""

    def __init__(self):
        from scrs_b200.api import Api, Library

        self.lib = load_oracle()
        self.api = Api(Library(ROOT / "oracle" / "_build" / "liboracle.so", prefix="oracle_", device=False))
        self.threads = int(self.lib.oracle_baseline_threads())
        self.gfni = bool(self.lib.oracle_simd_active())

    def time_stripes(self, desc, threads, target_s, min_passes=2, max_passes=200):
        """Median seconds of one pass of the host descriptors `desc`
        (DESC_DTYPE, host pointers) over `threads` threads, and the pass count."""
        st = C.c_int32()
        times = []
        t_end = time.perf_counter() + target_s
        while len(times) < min_passes or (time.perf_counter() < t_end and len(times) < max_passes):
            times.append(self.lib.oracle_baseline_stripes(desc.ctypes.data, len(desc), threads, C.byref(st)))
            if st.value:
                raise RuntimeError(f"oracle stripe baseline failed with status {st.value}")
        return float(np.median(times)), len(times)

    def codec_leg(self, op, engine, k, m, Ls, data, word, order, target_s=2.0):
        """One codec geometry on the host cores: every pass runs one
        independent stripe per host thread (the reference is single-threaded
        per codec) encoding `data` or decoding the received rows `order` of
        `word`; and one stripe on one thread.  Goodput counts k*L per stripe."""
        from scrs_b200.batch import DESC_DTYPE, OP_DECODE

        T = self.threads
        if op == OP_DECODE:
            src = np.ascontiguousarray(np.concatenate([word[i] for i in order]))
            outs = np.zeros((T, k * Ls), np.uint8)
            idx = np.ascontiguousarray(np.asarray(order, dtype=np.uint16))
        else:
            src = np.ascontiguousarray(data)
            outs = np.zeros((T, m * Ls), np.uint8)
            idx = None
        desc = np.zeros(T, dtype=DESC_DTYPE)
        desc["op"], desc["engine"], desc["k"], desc["m"], desc["symbol_len"] = op, int(engine), k, m, Ls
        desc["in_"] = src.ctypes.data
        desc["out"] = outs.ctypes.data + np.arange(T, dtype=np.uint64) * outs.shape[1]
        if idx is not None:
            desc["indices"] = idx.ctypes.data
        t_one, _ = self.time_stripes(desc[:1], 1, target_s / 4, min_passes=1, max_passes=20)
        t_all, passes = self.time_stripes(desc, T, target_s)
        ok = bool(np.array_equal(outs[0], outs[-1]))
        if op == OP_DECODE:
            ok &= bool(np.array_equal(outs[0], data))
        return {"GBps": round(T * k * Ls / t_all / 1e9, 3), "single_core_GBps": round(k * Ls / t_one / 1e9, 3),
                "single_core_ms": round(t_one * 1e3, 3), "cores": T, "passes": passes, "bit_exact": ok}

    def block(self, legs: dict, sample: str) -> dict:
        return {"kind": "port", "cores": self.threads, "cpu": host_cpu(),
                "sample": sample + f"; CPU restatement of the reference (oracle/, GFNI={'on' if self.gfni else 'off'})",
                **legs}


# ---------------------------------------------------------------------------
# extras: batched vs plain (config 4), latency, tower, AFFT, serving
# ---------------------------------------------------------------------------

def time_ms(torch, fn, reps):
    reps = reps if CALL_REPS is None else CALL_REPS
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def per_call_ms(torch, fn, samples=200, warm=5):
    """p50 / p99 of `samples` single calls, each bracketed by CUDA events on
    the current stream and synchronised (host issue cost included)."""
    if CALL_REPS is not None:
        samples, warm = CALL_REPS, 0
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(samples):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        ts.append(s.elapsed_time(e))
    return round(float(np.percentile(ts, 50)), 4), round(float(np.percentile(ts, 99)), 4)


def roofline_of(nbytes, ms, note):
    peak, kind = peaks()
    ach = nbytes / (ms / 1e3) / 1e9
    return {"bound": "hbm", "algorithmic_bytes": int(nbytes), "ms": round(ms, 4), "achieved": round(ach, 1),
            "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4), "peak_source": kind, "note": note}


def extra_mixed(torch, api, cpu=None):
    """Config 4: 8192 stripes, k~U[4,64], m~U[1,16], L in {1,4,64} KiB, half
    encode, half decode of real codewords (up to m data symbols erased),
    persistent+graph vs one launch per stripe.  Every decoded stripe is
    compared with its data, every repair with a separate encode pass, and a
    sample of each symbol length with the oracle."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import DESC_DTYPE, OP_DECODE, OP_ENCODE, StripeBatch

    rng = np.random.default_rng(SEED + 4)
    n = MIXED_STRIPES
    ks = rng.integers(4, 65, n)
    ms = rng.integers(1, 17, n)
    Ls = rng.choice([1024, 4096, 65536], n)
    eng = np.where(rng.integers(0, 2, n) == 1, int(Engine.STANDARD_CAUCHY), int(Engine.GOOD_CAUCHY))
    op = np.where(np.arange(n) % 2 == 0, OP_ENCODE, OP_DECODE)
    dec = op == OP_DECODE
    # every stripe's codeword (k data rows, then m repair rows), one buffer
    w_sz = (ks + ms) * Ls
    w_off = np.concatenate([[0], np.cumsum(w_sz)[:-1]]).astype(np.uint64)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(SEED + 4)
    words = torch.randint(0, 256, (int(w_sz.sum()),), dtype=torch.uint8, device="cuda", generator=gen)
    wp = np.uint64(words.data_ptr())
    enc_pass = StripeBatch(api.lib, n)
    enc_pass.set_arrays(np.full(n, OP_ENCODE), eng, ks, ms, Ls, wp + w_off,
                        wp + w_off + (ks * Ls).astype(np.uint64))
    enc_pass.run()
    torch.cuda.synchronize()
    del enc_pass
    idx = np.zeros((n, 64), np.uint16)
    for s in np.nonzero(dec)[0]:
        k, m = int(ks[s]), int(ms[s])
        e = int(rng.integers(0, min(k, m) + 1))
        erased = rng.choice(k, e, replace=False)
        keep = np.setdiff1d(np.arange(k), erased)
        reps = k + rng.choice(m, e, replace=False)
        idx[s, :k] = rng.permutation(np.concatenate([keep, reps]))
    # received rows of the decode stripes, gathered on the device
    r_sz = np.where(dec, ks * Ls, 0)
    r_off = np.concatenate([[0], np.cumsum(r_sz)[:-1]]).astype(np.uint64)
    rcv = torch.empty(int(r_sz.sum()), dtype=torch.uint8, device="cuda")
    idx_d = torch.from_numpy(idx.astype(np.int64)).cuda()
    for s in np.nonzero(dec)[0]:
        k, m, Lx, wo, ro = int(ks[s]), int(ms[s]), int(Ls[s]), int(w_off[s]), int(r_off[s])
        rcv[ro:ro + k * Lx].view(k, Lx).copy_(words[wo:wo + (k + m) * Lx].view(k + m, Lx)[idx_d[s, :k]])
    out_sz = np.where(op == OP_ENCODE, ms * Ls, ks * Ls)
    out_off = np.concatenate([[0], np.cumsum(out_sz)[:-1]]).astype(np.uint64)
    outbuf = torch.zeros(int(out_sz.sum()), dtype=torch.uint8, device="cuda")
    ins = np.where(dec, np.uint64(rcv.data_ptr()) + r_off, wp + w_off)
    b = StripeBatch(api.lib, n)
    b.set_arrays(op, eng, ks, ms, Ls, ins, np.uint64(outbuf.data_ptr()) + out_off, indices=idx)
    goodput = float((ks * Ls).sum())
    algo = float(np.where(op == OP_ENCODE, (ks + ms) * Ls, 2 * ks * Ls).sum())
    default = b.launch_params
    b.run(graph=True)
    torch.cuda.synchronize()
    t_default = time_ms(torch, lambda: b.run(graph=True), 10)
    tuned = b.autotune(reps=3)  # the graph is re-captured with the tuned launch
    b.run(graph=True)
    torch.cuda.synchronize()
    t_graph = time_ms(torch, lambda: b.run(graph=True), 10)
    launches_batched = b.last_launches
    outbuf.zero_()
    b.run_plain()
    torch.cuda.synchronize()
    t_plain = time_ms(torch, lambda: b.run_plain(), 2)
    launches_plain = b.last_launches
    b.check()
    # outputs of the plain form, then of the persistent form
    ok = True
    for form in ("plain", "persistent"):
        if form == "persistent":
            outbuf.zero_()
            b.run(graph=True)
        torch.cuda.synchronize()
        for s in range(n):
            k, m, Lx, wo, oo = int(ks[s]), int(ms[s]), int(Ls[s]), int(w_off[s]), int(out_off[s])
            exp = words[wo:wo + k * Lx] if dec[s] else words[wo + k * Lx:wo + (k + m) * Lx]
            if not torch.equal(outbuf[oo:oo + int(out_sz[s])], exp):
                ok = False
                break
    # a sample of every symbol length against the oracle
    checked = 0
    if cpu is not None:
        for Lx in (1024, 4096, 65536):
            for want_dec in (False, True):
                for s in np.nonzero((Ls == Lx) & (dec == want_dec))[0][:2]:
                    k, m, wo, oo = int(ks[s]), int(ms[s]), int(w_off[s]), int(out_off[s])
                    word = words[wo:wo + (k + m) * Lx].cpu().numpy().reshape(k + m, Lx)
                    p = cpu.api.resolve(Engine(int(eng[s])), k, m, Lx)
                    got = outbuf[oo:oo + int(out_sz[s])].cpu().numpy()
                    if want_dec:
                        exp = np.zeros(k * Lx, np.uint8)
                        cpu.api.batch_decoder(p).decode_into([(int(i), word[i]) for i in idx[s, :k]], exp)
                    else:
                        exp = np.zeros(m * Lx, np.uint8)
                        cpu.api.batch_encoder(p).encode_into(word[:k].reshape(-1), exp)
                    ok &= bool(np.array_equal(got, exp))
                    checked += 1
    res = {"workload": f"{n} stripes, k~U[4,64], m~U[1,16], L in {{1,4,64}} KiB, Standard/Good mixed, half encode "
                       "half decode of real codewords (random erasures <= m)",
           "persistent_graph_GBps": round(goodput / t_graph / 1e6, 1),
           "plain_per_stripe_GBps": round(goodput / t_plain / 1e6, 1),
           "speedup": round(t_plain / t_graph, 2),
           "persistent_ms": round(t_graph, 3), "plain_ms": round(t_plain, 3),
           "persistent_hbm_frac": round(algo / t_graph / 1e6 / peaks()[0], 3),
           "roofline": roofline_of(algo, t_graph, "plan launch + persistent drain (mxk_kernel), graph replay"),
           "autotune": {"default": {"seg_rows": default.seg_rows, "ctas_per_sm": default.ctas_per_sm,
                                    "persistent_ms": round(t_default, 3)},
                        "chosen": {"seg_rows": tuned.seg_rows, "ctas_per_sm": tuned.ctas_per_sm,
                                   "persistent_ms": round(t_graph, 3)}},
           "launches": {"persistent": launches_batched, "plain": launches_plain},
           "bit_exact": ok, "oracle_checked_stripes": checked,
           "checks": "every output of the plain and the persistent form against the data / a separate encode pass; "
                     "2 encode + 2 decode stripes of each symbol length against the oracle"}
    if cpu is not None:
        # the first stripes of the batch (same distribution), inputs copied to the host
        take, acc = [], 0
        for s in range(n):
            take.append(s)
            acc += int(ks[s] * Ls[s])
            if acc > 600 << 20:
                break
        take = np.array(take)
        h_in, h_out, desc = [], [], np.zeros(len(take), dtype=DESC_DTYPE)
        for q, s in enumerate(take):
            k, m, Lx = int(ks[s]), int(ms[s]), int(Ls[s])
            src = rcv[int(r_off[s]):int(r_off[s]) + k * Lx] if dec[s] else words[int(w_off[s]):int(w_off[s]) + k * Lx]
            h_in.append(src.cpu().numpy())
            h_out.append(np.zeros(int(out_sz[s]), np.uint8))
            desc[q] = (int(op[s]), int(eng[s]), k, m, Lx, h_in[-1].ctypes.data, h_out[-1].ctypes.data,
                       idx[s].ctypes.data if dec[s] else 0)
        order = np.lexsort((desc["symbol_len"], desc["m"], desc["k"], desc["engine"], desc["op"]))
        desc = desc[order]
        gp = float(sum(int(ks[s] * Ls[s]) for s in take))
        t_all, passes = cpu.time_stripes(desc, cpu.threads, 6.0)
        one = desc[::max(1, len(desc) // 64)]
        t_one, _ = cpu.time_stripes(one, 1, 1.0, min_passes=1, max_passes=3)
        gp_one = float((one["k"].astype(np.float64) * one["symbol_len"]).sum())
        cpu_ok = all(np.array_equal(h_out[q], outbuf[int(out_off[s]):int(out_off[s]) + int(out_sz[s])].cpu().numpy())
                     for q, s in enumerate(take[:64]))
        res["cpu_baseline"] = cpu.block(
            {"value": round(gp / t_all / 1e9, 3), "unit": "GB/s", "single_core_GBps": round(gp_one / t_one / 1e9, 3),
             "passes": passes, "bit_exact": bool(cpu_ok)},
            f"the first {len(take)} stripes of the batch ({gp / 1e6:.0f} MB of data, mixed encode/decode), "
            f"sorted by geometry, one contiguous range per thread; single core: every "
            f"{max(1, len(desc) // 64)}th of them")
    return res


def extra_latency(torch, api, cpu=None):
    """Single-stripe latency of config 1 through the per-codec device entry points."""
    from scrs_b200.api import Engine

    p = api.resolve(Engine.GOOD_CAUCHY, K, M, L)
    enc = api.batch_encoder(p)
    es = enc.scratch()
    data = torch.randint(0, 256, (K * L,), dtype=torch.uint8, device="cuda")
    rep = torch.zeros(M * L, dtype=torch.uint8, device="cuda")
    dec = api.batch_decoder(p)
    ds = dec.scratch()
    out = torch.zeros(K * L, dtype=torch.uint8, device="cuda")
    idx = [0, 2, 3, 5, 6, 8, 10, 11, 12, 13]
    enc.encode_into_with(data, rep, es)
    word = torch.cat([data.view(K, L), rep.view(M, L)])
    rows = word[torch.tensor(idx, device="cuda")].reshape(-1).contiguous()
    res = {}
    for name, fn in (("encode", lambda: enc.encode_into_with(data, rep, es)),
                     ("decode", lambda: dec.decode_into_with((idx, rows), out, ds))):
        res[f"{name}_p50_ms"], res[f"{name}_p99_ms"] = per_call_ms(torch, fn, warm=20)
    res["bit_exact"] = bool(torch.equal(out, data))
    res["workload"] = "one stripe k=10 m=4 L=4096, device buffers, per-call launch (encode: 1 kernel; decode: 1 kernel, the plan comes from the recipe cache after the first call)"
    return res


# offered Poisson arrival rates of the serving sweep, past the closed-loop capacity
RATES_PER_S = (2500.0, 5000.0, 10000.0, 20000.0, 30000.0, 40000.0, 60000.0)


def extra_serving(torch, api, cpu=None, seconds_per_rate=1.5, n_templates=192, seed=0x5C250005):
    """Config 5: Poisson arrivals of mixed encode/decode requests over all four
    engines through the serving loop (scrs_server_*), 64 GB budget, 8 slots.
    The closed-loop capacity (2000 requests submitted at once, median of five
    passes after a warm-up pass, each pass with a host timeline) is reported
    beside a sweep of fixed Poisson rates up to past that capacity, so that
    runs on different hosts compare at the same offered load.  Requests are
    192 templates of real codewords; after the sweep every template's output
    is compared with its expected bytes (the regular entry points' result,
    itself compared with the oracle for one template per engine).  Latency =
    completion seen by the host - submit.  Python's garbage collector is
    paused during the timed passes and rates: one of its collections stops
    this polling loop for milliseconds, which would show as server latency."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import DESC_DTYPE
    from scrs_b200.serving import OP_DECODE, OP_ENCODE, Server

    rng = np.random.default_rng(seed)
    tower = [(64, 16, 4096), (256, 64, 1024), (1024, 256, 512), (32, 8, 65536)]
    afft = [(1024, 1024, 1024), (4096, 4096, 256), (3000, 500, 2048), (16384, 16384, 256)]
    encoders = {}

    def encode(engine, k, m, Ls, data):
        key = (engine, k, m, Ls)
        p = api.resolve(engine, k, m, Ls)
        rep = torch.zeros(m * Ls, dtype=torch.uint8, device="cuda")
        if engine == Engine.TOWER:
            inc = encoders.get(key) or api.incremental_encoder(p)
            encoders[key] = inc
            inc.reset()
            for i in range(k):
                inc.feed(i, data[i * Ls:(i + 1) * Ls])
            for j in range(m):
                rep[j * Ls:(j + 1) * Ls].copy_(torch.frombuffer(bytearray(inc.repair(j)), dtype=torch.uint8))
        else:
            pair = encoders.get(key)
            if pair is None:
                e = api.batch_encoder(p)
                pair = encoders[key] = (e, e.scratch())
            pair[0].encode_into_with(data, rep, pair[1])
        return rep

    templates = []
    for t in range(n_templates):
        u = rng.random()
        if u < 0.7:
            engine = Engine.STANDARD_CAUCHY if rng.random() < 0.5 else Engine.GOOD_CAUCHY
            k = int(rng.integers(4, 65))
            m = int(rng.integers(1, 17))
            Ls = int(rng.choice([1024, 4096, 16384, 65536]))
        elif u < 0.85:
            engine = Engine.TOWER
            k, m, Ls = tower[int(rng.integers(0, len(tower)))]
        else:
            engine = Engine.AFFT
            k, m, Ls = afft[int(rng.integers(0, len(afft)))]
        op = OP_ENCODE if rng.random() < 0.5 else OP_DECODE
        data = torch.randint(0, 256, (k * Ls,), dtype=torch.uint8, device="cuda")
        rep = encode(engine, k, m, Ls, data)
        idx = None
        if op == OP_ENCODE:
            d_in, expect = data, rep
        else:
            e = int(rng.integers(0, min(k, m) + 1))
            erased = set(rng.choice(k, e, replace=False).tolist()) if e else set()
            idx = [i for i in range(k) if i not in erased] + [k + j for j in rng.choice(m, e, replace=False).tolist()]
            idx = np.asarray(idx, dtype=np.uint64)
            word = torch.cat([data.view(k, Ls), rep.view(m, Ls)])
            d_in = word[torch.from_numpy(idx.astype(np.int64)).cuda()].reshape(-1).contiguous()
            expect = data
        d_out = torch.zeros(expect.numel(), dtype=torch.uint8, device="cuda")
        templates.append((op, engine, k, m, Ls, d_in, d_out, idx, expect))
    encoders.clear()
    torch.cuda.synchronize()
    # the regular entry points' repairs against the oracle, one template per engine
    oracle_ok, oracle_checked = True, 0
    if cpu is not None:
        for want in (Engine.STANDARD_CAUCHY, Engine.GOOD_CAUCHY, Engine.TOWER, Engine.AFFT):
            for op, engine, k, m, Ls, d_in, d_out, idx, expect in templates:
                if engine == want and op == OP_ENCODE:
                    p = cpu.api.resolve(engine, k, m, Ls)
                    host = d_in.cpu().numpy()
                    if engine == Engine.TOWER:
                        inc = cpu.api.incremental_encoder(p)
                        for i in range(k):
                            inc.feed(i, host[i * Ls:(i + 1) * Ls])
                        exp = np.frombuffer(b"".join(inc.repair(j) for j in range(m)), np.uint8)
                    else:
                        exp = np.zeros(m * Ls, np.uint8)
                        cpu.api.batch_encoder(p).encode_into(host, exp)
                    oracle_ok &= bool(np.array_equal(expect.cpu().numpy(), exp))
                    oracle_checked += 1
                    break
    srv = Server(api.lib, 64 << 30, slots=8)
    # start-up: the tower and additive-FFT profiles' engines resident on every slot
    for op, engine, k, m, Ls, *_ in templates:
        if engine in (Engine.TOWER, Engine.AFFT):
            srv.reserve(op, engine, k, m, Ls)

    # each template built once as a request; a submit is then one library call
    prepared = [srv.prepare(op, engine, k, m, Ls, d_in.data_ptr(), d_out.data_ptr(), idx, tag=t)
                for t, (op, engine, k, m, Ls, d_in, d_out, idx, _) in enumerate(templates)]
    goodput_of = np.array([tp[2] * tp[4] for tp in templates], dtype=np.float64)

    def submit(t, tag):
        srv.submit_prepared(prepared[t])

    # warm the slots' stripe-batch buffers (a closed-loop pass coalesces larger
    # GF(256) groups than the template rounds, and the buffers grow, allocating,
    # until they fit), then the closed-loop capacity
    for _ in range(8):
        for t in range(len(templates)):
            submit(t, t)
        srv.drain(600)
    passes = []  # closed loop: one warm-up pass, then 5 passes of 2000 requests submitted at once, median kept
    gc.collect()
    gc.disable()
    for p in range(6):
        order = rng.integers(0, len(templates), 2000)
        b0 = srv.stats()["batches"]
        t0 = time.perf_counter()
        for t in order:
            submit(int(t), int(t))
        t_sub = time.perf_counter()
        calls, slowest = 0, 0.0
        while srv.pending:
            c0 = time.perf_counter()
            srv.progress()
            c1 = time.perf_counter()
            calls += 1
            slowest = max(slowest, c1 - c0)
            if c1 - t0 > 600:
                raise TimeoutError("closed-loop pass did not drain")
        cap_s = time.perf_counter() - t0
        if p:
            passes.append({"requests_per_s": round(len(order) / cap_s, 1),
                           "goodput_GBps": round(sum(templates[int(t)][2] * templates[int(t)][4] for t in order)
                                                 / cap_s / 1e9, 2),
                           "submit_ms": round((t_sub - t0) * 1e3, 2), "drain_ms": round((cap_s - (t_sub - t0)) * 1e3, 2),
                           "progress_calls": calls, "slowest_progress_ms": round(slowest * 1e3, 2),
                           "batches": srv.stats()["batches"] - b0})
    med = sorted(passes, key=lambda x: x["requests_per_s"])[len(passes) // 2]
    res = {"workload": "Poisson arrivals; 70% GF(256) (Standard/Good, k~U[4,64], m~U[1,16], L in {1,4,16,64} KiB), "
                       "15% tower (k<=1024, m<=256), 15% AFFT (k<=16384, m<=16384, L 256-2048); half encode, half "
                       "decode of real codewords with random erasures <= m; 64 GB budget, 8 slots, GF(256) coalesced "
                       "per slot",
           "closed_loop": {"requests_per_s": med["requests_per_s"], "goodput_GBps": med["goodput_GBps"],
                           "passes": passes},
           "rates": []}
    for rate in RATES_PER_S:
        n = int(rate * seconds_per_rate)
        arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
        picks = rng.integers(0, len(templates), n)
        chunks, i = [], 0
        t0 = time.perf_counter()
        while i < n or srv.pending:
            now = time.perf_counter() - t0
            while i < n and arrivals[i] <= now:
                srv.submit_prepared(prepared[picks[i]])
                i += 1
            got = srv.progress_arrays()
            if len(got[0]):
                chunks.append(got)
        el = time.perf_counter() - t0
        tags = np.concatenate([c[0] for c in chunks]).astype(np.int64)
        status = np.concatenate([c[1] for c in chunks])
        lat = (np.concatenate([c[3] for c in chunks]) - np.concatenate([c[2] for c in chunks])) / 1e6
        gb = float(goodput_of[tags].sum())
        res["rates"].append({"offered_per_s": round(rate, 1), "requests": n, "achieved_per_s": round(n / el, 1),
                             "failed": int((status != 0).sum()),
                             "goodput_GBps": round(gb / el / 1e9, 2), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                             "p99_ms": round(float(np.percentile(lat, 99)), 3)})
        gc.collect()  # between rates, outside the timed loop
    gc.enable()
    # The timed phases submit templates again while earlier requests of the
    # same template are in flight, so requests share output buffers there and
    # their bytes prove nothing.  The check: every template once, all at once
    # (coalesced and overlapping as in the mix, but each output written by one
    # request), against its expected bytes.
    for t in templates:
        t[6].zero_()
    torch.cuda.synchronize()
    for t in range(len(templates)):
        submit(t, t)
    final = srv.drain(600)
    torch.cuda.synchronize()
    res["stats"] = srv.stats()
    srv.close()
    wrong = [t for t in templates if not torch.equal(t[6], t[8])]
    wrong += [templates[c.tag] for c in final if c.status != 0]
    outputs_ok = not wrong
    res["bit_exact"] = bool(outputs_ok and oracle_ok)
    if not res["bit_exact"]:  # which templates, for the record
        res["mismatches"] = {"oracle_ok": bool(oracle_ok),
                             "templates": [{"op": int(t[0]), "engine": Engine(t[1]).name, "k": t[2], "m": t[3],
                                            "L": t[4],
                                            "bytes_differing": int((t[6] != t[8]).sum().item())} for t in wrong[:8]],
                             "count": len(wrong)}
    res["checks"] = (f"after the sweep, all {len(templates)} templates submitted at once, each output equal to its "
                     f"expected bytes (the regular entry points' result); {oracle_checked} encode templates' expected "
                     "bytes equal the oracle's")
    if cpu is not None:
        # the template mix once per pass on the host cores (one contiguous range per thread)
        h_in, h_out, desc = [], [], np.zeros(len(templates), dtype=DESC_DTYPE)
        h_idx = []
        for q, (op, engine, k, m, Ls, d_in, d_out, idx, expect) in enumerate(templates):
            h_in.append(d_in.cpu().numpy())
            h_out.append(np.zeros(expect.numel(), np.uint8))
            h_idx.append(np.asarray(idx if idx is not None else [0], dtype=np.uint16))
            desc[q] = (op, int(engine), k, m, Ls, h_in[-1].ctypes.data, h_out[-1].ctypes.data,
                       h_idx[-1].ctypes.data if op == OP_DECODE else 0)
        desc = desc[np.lexsort((desc["symbol_len"], desc["m"], desc["k"], desc["engine"], desc["op"]))]
        gp = float((desc["k"].astype(np.float64) * desc["symbol_len"]).sum())
        t_all, passes_cpu = cpu.time_stripes(desc, cpu.threads, 4.0, min_passes=1)
        res["cpu_baseline"] = cpu.block(
            {"value": round(gp / t_all / 1e9, 3), "unit": "GB/s", "passes": passes_cpu,
             "requests_per_s": round(len(desc) / t_all, 1)},
            f"the {len(templates)} request templates once per pass, sorted by geometry, one contiguous range "
            "per thread (no arrivals: the host cores' throughput on the same mix)")
    return res


def extra_tower(torch, api, cpu=None):
    """Config 2: Tower k=32 m=8 L=65536, incremental encode (32 feeds) + lazy decode (8 data erased)."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import OP_DECODE, OP_ENCODE

    k, m, Lt = 32, 8, 65536
    p = api.resolve(Engine.TOWER, k, m, Lt)
    inc = api.incremental_encoder(p)
    dec = api.decoder(p)
    ds = dec.scratch()
    data = torch.randint(0, 256, (k, Lt), dtype=torch.uint8, device="cuda")
    out = torch.zeros(k * Lt, dtype=torch.uint8, device="cuda")

    rows = [data[i] for i in range(k)]  # row views made once, outside the timed calls

    def encode():
        inc.reset()
        for i in range(k):
            inc.feed(i, rows[i])
        inc.repair_device_ptr(0)  # folds pending feeds, waits for the encoder's stream

    encode()
    reps = [torch.empty(Lt, dtype=torch.uint8, device="cuda") for _ in range(m)]
    for j in range(m):
        reps[j].copy_(torch.frombuffer(bytearray(inc.repair(j)), dtype=torch.uint8).cuda())
    rng = np.random.default_rng(SEED + 2)
    erased = set(rng.choice(k, 8, replace=False).tolist())
    order = [i for i in rng.permutation(k + m).tolist() if i not in erased][:k]
    word = [data[i] for i in range(k)] + reps

    def decode():
        dec.reset()
        for i in order:
            dec.push(i, word[i])
        dec.finalize_into_with(out, ds)

    decode()
    torch.cuda.synchronize()
    ok = bool(torch.equal(out.view(k, Lt), data))
    t_enc = time_ms(torch, encode, 10)
    t_dec = time_ms(torch, decode, 10)
    e50, e99 = per_call_ms(torch, encode)
    d50, d99 = per_call_ms(torch, decode)
    res = {"workload": "Tower k=32 m=8 L=65536: 32 device feeds + repair fold; lazy decode r=8 (32 device pushes + "
                       "finalize)",
           "encode_GBps": round(k * Lt / t_enc / 1e6, 1), "decode_GBps": round(k * Lt / t_dec / 1e6, 1),
           "encode_ms": round(t_enc, 3), "decode_ms": round(t_dec, 3),
           "encode_p50_ms": e50, "encode_p99_ms": e99, "decode_p50_ms": d50, "decode_p99_ms": d99,
           "roofline": {"encode": roofline_of((k + m) * Lt, t_enc, "32 feeds + one fold launch, per call"),
                        "decode": roofline_of(2 * k * Lt, t_dec, "32 pushes + plan + multiply-XOR, per call")}}
    res["batched"] = tower_batched(torch, api, k, m, Lt, np.concatenate([r.cpu().numpy() for r in reps]),
                                   data.cpu().numpy().reshape(-1))
    ok &= res["batched"]["bit_exact"]
    if cpu is not None:
        h_data = data.cpu().numpy().reshape(-1)
        h_word = [w.cpu().numpy() for w in word]
        exp = np.frombuffer(b"".join(cpu_encode_tower(cpu, p, h_data)), np.uint8)
        ok &= bool(np.array_equal(np.concatenate(h_word[k:]), exp))
        legs = {"encode": cpu.codec_leg(OP_ENCODE, Engine.TOWER, k, m, Lt, h_data, h_word, order),
                "decode": cpu.codec_leg(OP_DECODE, Engine.TOWER, k, m, Lt, h_data, h_word, order)}
        res["cpu_baseline"] = cpu.block(legs, "one stripe per host thread per pass: 32 in-order feeds + 8 repair "
                                              "reads (encode), batch decode of the same 32 received symbols (decode)")
        ok &= legs["encode"]["bit_exact"] and legs["decode"]["bit_exact"]
    res["bit_exact"] = ok
    return res


def tower_batched(torch, api, k, m, Lt, rep0, data0, n=128, seed=SEED + 22):
    """The cfg2 geometry as stripes of one batch: n tower encodes and n tower
    decodes (8 data symbols erased each, random arrival order) in one plan
    launch + one persistent drain, replayed as a CUDA graph.  Stripe 0's
    data is the per-call extra's, so its repairs are checked against the
    incremental encoder's; every decode against its data."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import OP_DECODE, OP_ENCODE, StripeBatch

    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    data = torch.randint(0, 256, (n, k * Lt), dtype=torch.uint8, device="cuda", generator=gen)
    data[0].copy_(torch.from_numpy(data0))
    reps = torch.zeros((n, m * Lt), dtype=torch.uint8, device="cuda")
    eng = int(Engine.TOWER)
    b = StripeBatch(api.lib, 2 * n)
    idx = np.arange(n, dtype=np.uint64)
    b.set_arrays(np.full(n, OP_ENCODE), np.full(n, eng), np.full(n, k), np.full(n, m), np.full(n, Lt),
                 data.data_ptr() + idx * (k * Lt), reps.data_ptr() + idx * (m * Lt))
    b.run()
    torch.cuda.synchronize()
    ok = bool(np.array_equal(reps[0].cpu().numpy(), rep0))
    rng = np.random.default_rng(seed)
    recv = np.zeros((n, k), np.int64)
    for s in range(n):
        erased = set(rng.choice(k, 8, replace=False).tolist())
        recv[s] = [i for i in rng.permutation(k + m).tolist() if i not in erased][:k]
    word = torch.cat([data.view(n, k, Lt), reps.view(n, m, Lt)], dim=1)
    received = word[torch.arange(n, device="cuda")[:, None], torch.from_numpy(recv).cuda()].reshape(n, k * Lt)
    del word
    out = torch.zeros((n, k * Lt), dtype=torch.uint8, device="cuda")
    enc_out = torch.zeros_like(reps)
    op = np.concatenate([np.full(n, OP_ENCODE), np.full(n, OP_DECODE)])
    ins = np.concatenate([data.data_ptr() + idx * (k * Lt), received.data_ptr() + idx * (k * Lt)])
    outs = np.concatenate([enc_out.data_ptr() + idx * (m * Lt), out.data_ptr() + idx * (k * Lt)])
    indices = np.zeros((2 * n, k), np.uint16)
    indices[n:] = recv
    b.set_arrays(op, np.full(2 * n, eng), np.full(2 * n, k), np.full(2 * n, m), np.full(2 * n, Lt), ins, outs,
                 indices=indices)
    b.run(graph=True)
    torch.cuda.synchronize()
    ok &= bool(torch.equal(out, data)) and bool(torch.equal(enc_out, reps))
    t = time_ms(torch, lambda: b.run(graph=True), 10)
    goodput = 2 * n * k * Lt
    algo = n * (k + m) * Lt + n * 2 * k * Lt
    return {"workload": f"{n} tower encodes + {n} tower decodes (k={k} m={m} L={Lt}, 8 data symbols erased) in one "
                        "stripe batch: plan launch + persistent drain (mxk_kernel<1>), CUDA graph",
            "GBps": round(goodput / t / 1e6, 1), "ms": round(t, 3), "launches": b.last_launches,
            "roofline": roofline_of(algo, t, "tower plan + persistent tower drain"), "bit_exact": ok}


def cpu_encode_tower(cpu, p, h_data):
    inc = cpu.api.incremental_encoder(p)
    Ls = p.symbol_len
    for i in range(p.k):
        inc.feed(i, h_data[i * Ls:(i + 1) * Ls])
    return [inc.repair(j) for j in range(p.m)]


def extra_afft(torch, api, cpu=None):
    """Config 3: additive FFT k=4096 m=4096 L=1024 and k=32768 m=16384 L=256.
    Each mean is over 20 back-to-back calls between CUDA events on the
    stream (a call's host work overlaps the device work of the calls
    before); p50 / p99 are over 200 single calls.  Repairs are compared with
    the oracle's, decodes with the data."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import OP_DECODE, OP_ENCODE

    res = {}
    for tag, k, m, La in (("3a", 4096, 4096, 1024), ("3b", 32768, 16384, 256)):
        p = api.resolve(Engine.AFFT, k, m, La)
        enc = api.batch_encoder(p)
        es = enc.scratch()
        data = torch.randint(0, 256, (k * La,), dtype=torch.uint8, device="cuda")
        rep = torch.zeros(m * La, dtype=torch.uint8, device="cuda")
        enc.encode_into_with(data, rep, es)
        torch.cuda.synchronize()
        t_enc = time_ms(torch, lambda: enc.encode_into_with(data, rep, es), 20)
        e50, e99 = per_call_ms(torch, lambda: enc.encode_into_with(data, rep, es))
        sel = np.sort(np.random.default_rng(SEED + 3).permutation(k + m)[:k])
        word = torch.cat([data.view(k, La), rep.view(m, La)])
        rows = word[torch.from_numpy(sel).cuda()].reshape(-1).contiguous()
        dec = api.batch_decoder(p)
        ds = dec.scratch()
        out = torch.zeros(k * La, dtype=torch.uint8, device="cuda")
        sel64 = sel.astype(np.uint64)
        dec.decode_into_with((sel64, rows), out, ds)
        torch.cuda.synchronize()
        ok = bool(torch.equal(out, data))
        t_dec = time_ms(torch, lambda: dec.decode_into_with((sel64, rows), out, ds), 20)
        d50, d99 = per_call_ms(torch, lambda: dec.decode_into_with((sel64, rows), out, ds))
        # few erasures (2 data symbols lost): the targeted path
        few = np.array(list(range(2, k)) + [k, k + 1], dtype=np.uint64)
        rows2 = word[torch.from_numpy(few.astype(np.int64)).cuda()].reshape(-1).contiguous()
        out.zero_()
        dec.decode_into_with((few, rows2), out, ds)
        torch.cuda.synchronize()
        ok &= bool(torch.equal(out, data))
        t_few = time_ms(torch, lambda: dec.decode_into_with((few, rows2), out, ds), 20)
        f50, f99 = per_call_ms(torch, lambda: dec.decode_into_with((few, rows2), out, ds))
        r = {"k": k, "m": m, "symbol_len": La, "encode_GBps": round(k * La / t_enc / 1e6, 2),
             "decode_GBps": round(k * La / t_dec / 1e6, 2), "encode_ms": round(t_enc, 3),
             "decode_ms": round(t_dec, 3), "decode_2_erasures_ms": round(t_few, 3),
             "decode_2_erasures_GBps": round(k * La / t_few / 1e6, 2),
             "encode_p50_ms": e50, "encode_p99_ms": e99, "decode_p50_ms": d50, "decode_p99_ms": d99,
             "decode_2_erasures_p50_ms": f50, "decode_2_erasures_p99_ms": f99,
             "roofline": {"encode": roofline_of((k + m) * La, t_enc, "butterfly passes (afft_tile_kernel), "
                                                                     "slicing and unslicing fused into the first and last pass"),
                          "decode": roofline_of(2 * k * La, t_dec, "locator + transforms + derivative"),
                          "ncu_summary": "profiles/afft_cfg3_launches.md"}}
        if cpu is not None:
            h_data = data.cpu().numpy()
            h_rep = rep.cpu().numpy()
            exp = np.zeros(m * La, np.uint8)
            cpu.api.batch_encoder(cpu.api.resolve(Engine.AFFT, k, m, La)).encode_into(h_data, exp)
            ok &= bool(np.array_equal(h_rep, exp))
            h_word = list(h_data.reshape(k, La)) + list(h_rep.reshape(m, La))
            legs = {"encode": cpu.codec_leg(OP_ENCODE, Engine.AFFT, k, m, La, h_data, h_word, None),
                    "decode": cpu.codec_leg(OP_DECODE, Engine.AFFT, k, m, La, h_data, h_word, sel.tolist())}
            r["cpu_baseline"] = cpu.block(legs, "one stripe per host thread per pass: block encode (encode); batch "
                                                "decode of the same random half of the symbols (decode)")
            ok &= legs["encode"]["bit_exact"] and legs["decode"]["bit_exact"]
        r["bit_exact"] = ok
        res[tag] = r
    return res


def extra_sweep(torch, api, cpu=None, ks=(10, 32, 64), ms=(4, 8, 16), Ls=4096, in_bytes=None):
    """The GF(256) envelope: for each (k, m), a batch of Good Cauchy stripes
    (L = 4 KiB, enough stripes for about 512 MB of input, far above L2) run
    as encodes and, separately, as batch decodes from seeded random k-of-n
    receipt sets, each as one persistent launch.  Per cell: the drain's
    CUDA-event time (plan launch excluded), its algorithmic bytes ((k+m)*L per
    encode, 2*k*L per decode) and HBM fraction, and which drain ran (the
    matrix-specialised encode kernel where eligible)."""
    from scrs_b200.api import Engine
    from scrs_b200.batch import OP_DECODE, OP_ENCODE, StripeBatch

    peak = peaks()[0]
    eng = int(Engine.GOOD_CAUCHY)
    in_bytes = ENVELOPE_BYTES if in_bytes is None else in_bytes
    grid = ENVELOPE_CELLS or [(k, m) for k in ks for m in ms]
    cells, ok = [], True
    for k, m in grid:
        n = max(1, in_bytes // (k * Ls))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(SEED + 100 + k * 17 + m)
        data = torch.randint(0, 256, (n, k * Ls), dtype=torch.uint8, device="cuda", generator=gen)
        reps = torch.zeros((n, m * Ls), dtype=torch.uint8, device="cuda")
        idx = np.arange(n, dtype=np.uint64)
        b = StripeBatch(api.lib, n)
        b.set_arrays(np.full(n, OP_ENCODE), np.full(n, eng), np.full(n, k), np.full(n, m), np.full(n, Ls),
                     data.data_ptr() + idx * (k * Ls), reps.data_ptr() + idx * (m * Ls))
        b.run()
        torch.cuda.synchronize()
        enc = [b.run_timed_drains() for _ in range(5)]
        t_enc = float(np.median([r[1] + r[2] for r in enc]))
        spec = b.jit_stripes > 0
        rng = np.random.default_rng(SEED + 200 + k * 17 + m)
        recv = np.argsort(rng.random((n, k + m)), axis=1)[:, :k].astype(np.int64)
        word = torch.cat([data.view(n, k, Ls), reps.view(n, m, Ls)], dim=1)
        received = word[torch.arange(n, device="cuda")[:, None], torch.from_numpy(recv).cuda()].reshape(n, k * Ls)
        del word
        out = torch.zeros((n, k * Ls), dtype=torch.uint8, device="cuda")
        b.set_arrays(np.full(n, OP_DECODE), np.full(n, eng), np.full(n, k), np.full(n, m), np.full(n, Ls),
                     received.data_ptr() + idx * (k * Ls), out.data_ptr() + idx * (k * Ls),
                     indices=recv.astype(np.uint16))
        b.run()
        torch.cuda.synchronize()
        ok &= bool(torch.equal(out, data))
        dec = [b.run_timed_drains() for _ in range(5)]
        t_dec = float(np.median([r[2] for r in dec]))
        plan = float(np.median([r[0] for r in dec]))
        b.check()
        enc_bytes, dec_bytes = n * (k + m) * Ls, n * 2 * k * Ls
        cells.append({"k": k, "m": m, "stripes": n,
                      "encode_ms": round(t_enc, 4), "encode_frac": round(enc_bytes / t_enc / 1e6 / peak, 3),
                      "encode_kernel": "scrs_spec_drain" if spec else "mxk_kernel<0>",
                      "decode_ms": round(t_dec, 4), "decode_frac": round(dec_bytes / t_dec / 1e6 / peak, 3),
                      "decode_plan_ms": round(plan, 4),
                      "mean_erased": round(float((recv >= k).sum()) / n, 2)})
        del data, reps, received, out, b
        torch.cuda.empty_cache()
    return {"workload": "Good Cauchy stripes, L=4096, ~512 MB of input per cell; encode and batch decode (seeded "
                        "random k-of-n receipt sets) as persistent launches; drain time by CUDA events",
            "peak_GBps": peak, "cells": cells, "bit_exact": ok}


EXTRAS = {"batched_vs_plain_cfg4": extra_mixed, "gf256_envelope": extra_sweep, "latency_cfg1": extra_latency, "tower_cfg2": extra_tower,
          "afft_cfg3": extra_afft, "serving_cfg5": extra_serving}


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------

def run_ours(args, world, rank, local):
    import torch

    torch.cuda.set_device(local)
    import scrs_b200
    from scrs_b200.api import Api, Library

    api = scrs_b200.api_default()
    w = build_cfg1(torch, api, rank)
    b = w["batch"]
    tuned = b.autotune(reps=3)  # launch parameters of the drain, chosen before any timing
    for _ in range(max(args.warmup, 3)):
        b.run(graph=True)
    torch.cuda.synchronize()
    oracle_api = None
    if rank == 0:
        subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
        oracle_api = Api(Library(ROOT / "oracle" / "_build" / "liboracle.so", prefix="oracle_", device=False))
    ok = verify_cfg1(torch, api, w, oracle_api)
    # ---- timed region: K graph replays, events on the launching stream
    stream = torch.cuda.current_stream()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        for _ in range(args.steps):
            b.run(stream, graph=True)
        e.record(stream)
        torch.cuda.synchronize()
    b.check()
    barrier(world)
    ms = barrier_max(s.elapsed_time(e) / args.steps, world)
    launches = b.last_launches * args.steps
    value = goodput_bytes() * world / (ms / 1e3) / 1e9
    # ---- roofline of the drain (events around the drain launches only): the
    # encode stripes run through the kernel specialised to the k=10 m=4 Good
    # Cauchy matrix, the decode stripes through the generic drain
    runs = [b.run_timed_drains() for _ in range(max(5, min(20, args.steps)))]
    spec_ms = float(np.mean([r[1] for r in runs]))
    gen_ms = float(np.mean([r[2] for r in runs]))
    drain_ms = spec_ms + gen_ms
    peak, peak_kind = peaks()
    achieved = algorithmic_bytes() / (drain_ms / 1e3) / 1e9
    ratio = profile_traffic_ratio()
    enc_spec = b.jit_stripes  # encode stripes on the specialised kernel (0 or all of them)
    spec_bytes = enc_spec * (K + M) * L
    gen_bytes = algorithmic_bytes() - spec_bytes

    def part(nbytes, ms):
        ach = nbytes / (ms / 1e3) / 1e9 if ms > 0 else 0.0
        return {"ms": round(ms, 4), "algorithmic_bytes": nbytes, "achieved": round(ach, 1),
                "frac": round(ach / peak, 4)}

    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if
            peak_kind == "measured" else "fallback 6650 GB/s",
            "traffic": round(ratio * algorithmic_bytes()) if ratio else None,
            "traffic_source": ("DRAM bytes per algorithmic byte of a 1-pass ncu capture of the full-size "
                               "65536+65536-stripe launches (dram__bytes_read.sum + dram__bytes_write.sum, "
                               "profiles/gf256_mxk_cfg1_ncu.md) times this launch's algorithmic bytes"),
            "kernel": ("persistent drain: scrs_spec_drain (encode stripes, kernel specialised to the matrix) "
                       "then mxk_kernel<0, 7> (decode stripes; rows 16-byte aligned, whole 2 KiB chunks, "
                       "one segment)" if enc_spec else "mxk_kernel<0, 7> persistent drain"),
            "algorithmic_bytes_per_launch": algorithmic_bytes(), "kernel_ms": round(drain_ms, 4),
            "parts": {"scrs_spec_drain": part(spec_bytes, spec_ms), "mxk_kernel<0, 7>": part(gen_bytes, gen_ms)}}
    # ---- e2e through the host-buffer batch entry point
    e2e = None
    if not args.no_e2e:
        from scrs_b200.api import Engine
        from scrs_b200.batch import OP_DECODE, OP_ENCODE, StripeBatch

        S = STRIPES
        h_in = torch.empty((2 * S, K * L), dtype=torch.uint8).pin_memory()
        h_in[:S].copy_(w["data"])
        h_in[S:].copy_(w["received"])
        h_rep = torch.empty((S, M * L), dtype=torch.uint8).pin_memory()
        h_dec = torch.empty((S, K * L), dtype=torch.uint8).pin_memory()
        del w["received"]
        hb = StripeBatch(api.lib, 2 * S)
        idx = np.arange(S, dtype=np.uint64)
        indices = np.zeros((2 * S, K), np.uint16)
        indices[S:] = w["recv"]
        hb.set_arrays(np.concatenate([np.full(S, OP_ENCODE), np.full(S, OP_DECODE)]),
                      np.full(2 * S, int(Engine.GOOD_CAUCHY)), np.full(2 * S, K), np.full(2 * S, M),
                      np.full(2 * S, L), h_in.data_ptr() + np.arange(2 * S, dtype=np.uint64) * (K * L),
                      np.concatenate([h_rep.data_ptr() + idx * (M * L), h_dec.data_ptr() + idx * (K * L)]),
                      indices=indices, host=True)
        hb.run(stream, graph=True)
        torch.cuda.synchronize()
        ok &= bool(torch.equal(h_dec, w["data"].cpu()))
        n_e2e = max(3, min(10, args.steps // 10))
        barrier(world)
        s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s2.record(stream)
        for _ in range(n_e2e):
            hb.run(stream, graph=True)
        e2.record(stream)
        torch.cuda.synchronize()
        ms_e2e = barrier_max(s2.elapsed_time(e2) / n_e2e, world)
        erased_rows = int((w["recv"] >= K).sum())  # r per decode stripe, summed
        link = h2d_rate(torch, h_in)
        e2e = {"value": round(goodput_bytes() * world / (ms_e2e / 1e3) / 1e9, 2), "unit": "GB/s",
               "h2d_bytes_per_step": 2 * S * K * L, "d2h_bytes_per_step": S * M * L + erased_rows * L,
               "ms_per_step": round(ms_e2e, 3), "steps": n_e2e,
               "link_bound": {"h2d_alone_GBps": round(link, 2),
                              "note": "goodput bytes equal host-to-device bytes on this workload (k*L in per "
                                      "stripe), so e2e cannot exceed the host-to-device copy rate measured alone "
                                      "(1 GiB pinned copy, CUDA events)"},
               "path": "scrs_stripe_batch_set_host + scrs_stripe_batch_run (pinned host buffers; copies of "
                       "64 pieces overlap the compute, both copy directions at once; decode stripes copy back "
                       "only their missing rows, their present rows are copied host-side while the GPU runs)"}
        launches += hb.last_launches * n_e2e
    extras = {}
    # the extras and the CPU baseline are single-GPU figures: taken at N = 1
    # only, so a multi-GPU run holds its GPUs for the headline alone
    if rank == 0 and world == 1 and not args.no_extras:
        cpu_legs = None if args.no_cpu else Cpu()
        for name, fn in EXTRAS.items():
            try:
                extras[name] = fn(torch, api, cpu_legs)
            except Exception as ex:  # reported, never hidden
                extras[name] = {"error": repr(ex)[:300]}
    if rank != 0:
        return
    cpu = None if args.no_cpu or world > 1 else cpu_baseline()
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic: seeded uniform random bytes (torch.Generator), seeded 10-of-14 erasure sets",
        "config": bench_config(world),
        "bit_exact": ok,
        "drain_launch": {"seg_rows": tuned.seg_rows, "ctas_per_sm": tuned.ctas_per_sm,
                         "chosen_by": "scrs_stripe_batch_autotune",
                         "encode_stripes_on_specialised_kernel": b.jit_stripes},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.result, "extras": extras,
    }
    print(json.dumps(line))


def run_reference(args, world, rank):
    if rank != 0:
        return
    lib = load_oracle()
    cal = CpuSample(lib, 256)
    t = min(cal.step() for _ in range(2))
    total_budget = 90.0
    per_step = total_budget / max(1, args.steps + args.warmup)
    count = int(max(64, min(STRIPES, 256 * per_step / max(t, 1e-6))))
    samp = CpuSample(lib, count)
    for _ in range(args.warmup):
        samp.step()
    times = [samp.step() for _ in range(args.steps)]
    dt = float(np.mean(times))
    value = samp.goodput_bytes() / dt / 1e9
    cpu = {"value": round(value, 3), "unit": "GB/s", "cores": samp.threads, "kind": "port",
           "sample": f"{count} stripes encoded + {count} batch-decoded per step (k=10 m=4 L=4096); CPU restatement "
                     f"of the reference (the Rust crate cannot be built: no cargo), GFNI="
                     f"{'on' if lib.oracle_simd_active() else 'off'}, {samp.threads} threads"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic: seeded uniform random bytes",
        "config": bench_config(world),
        "cpu_baseline": cpu, "e2e": {"value": round(value, 3), "unit": "GB/s", "h2d_bytes_per_step": 0,
                                     "d2h_bytes_per_step": 0}}))


def main():
    global STRIPES, MIXED_STRIPES, ENVELOPE_CELLS, ENVELOPE_BYTES, CALL_REPS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg (profiling runs)")
    ap.add_argument("--stripes", type=int, default=STRIPES,
                    help="stripes per op per GPU; the headline uses 65536, smaller values are for ncu captures")
    ap.add_argument("--mixed-stripes", type=int, default=MIXED_STRIPES,
                    help="stripes of the mixed batch extra; the reported figure uses 8192, smaller values are for ncu "
                         "captures")
    ap.add_argument("--envelope-cells", default=None,
                    help="GF(256) envelope cells as KxM[,KxM...] (default: the full sweep); for ncu captures")
    ap.add_argument("--envelope-mb", type=int, default=ENVELOPE_BYTES >> 20,
                    help="input MB per envelope cell (default 512; keep above the 126 MB L2)")
    ap.add_argument("--call-reps", type=int, default=None,
                    help="calls per mean and per percentile in the per-call extras (default 20 / 200); small "
                         "values keep ncu launch lists short")
    ap.add_argument("--only", choices=sorted(EXTRAS),
                    help="run just one of the extras and print its JSON (profiling runs; no headline line)")
    args = ap.parse_args()
    STRIPES = args.stripes
    MIXED_STRIPES = args.mixed_stripes
    if args.envelope_cells:
        ENVELOPE_CELLS = [tuple(int(v) for v in c.split("x")) for c in args.envelope_cells.split(",")]
    ENVELOPE_BYTES = args.envelope_mb << 20
    CALL_REPS = args.call_reps
    if args.only:
        import torch
        import scrs_b200

        print(json.dumps({args.only: EXTRAS[args.only](torch, scrs_b200.api_default())}))
        return
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
