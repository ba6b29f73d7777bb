"""Benchmark: RS(10,4) Gf8D encode + reconstruct of a batch of device-resident
stripes (256 stripes x 1 MiB shards), through the batched C-ABI path.

One step = one batched `dot_product_matrix_with` submission that encodes every
stripe (10 data shards -> 4 parity shards, Cauchy matrix c[i][j] =
inv(x_i + y_j), x_i = 10 + i, y_j = j) followed by one batched submission that
rebuilds 4 seeded-random erased shards of every stripe in place from 10
survivors (decode plans from host Gauss-Jordan inversion, cached per erasure
pattern). The rebuild is `mul_add_matrix_scattered` into rows that must be
zeroed first; it runs as the fused overwrite form of that op
(dot_product_matrix_scattered_with), which gives the same bytes without a
separate memset pass. The metric is source GB/s: the source bytes both
operations read (10 shards each, per stripe) per second, whole job.

Beside the headline the line carries the other measured configurations
(single 64 KiB stripe, 64 MiB shards, 256 MiB mul_add / scatter / gather,
the tower and large k*m shapes, the 4096-stripe mixed batch and the serving
loop), each checked against the oracle before it is timed.

python bench.py [--gpus N --steps K --warmup W] [--impl reference]
Under torchrun each rank runs its own batch (weak scaling, no collective on
the data path); time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RS(10,4) Gf8D encode+reconstruct source GB/s (batched, device-resident)"
K_SRC, M_PAR, N_ALL = 10, 4, 14
FALLBACK_HBM_GBS = 6650.0
MIB = 1 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--stripes", type=int, default=256)
    p.add_argument("--shard-mib", type=float, default=1.0)
    p.add_argument("--cpu-seconds", type=float, default=10.0, help="bounded CPU baseline sample")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-legs", action="store_true", help="skip the other configurations")
    p.add_argument("--no-uneven", action="store_true", help="skip the mixed-geometry batch comparison")
    p.add_argument("--uneven-stripes", type=int, default=4096)
    p.add_argument("--no-serve", action="store_true", help="skip the serving-loop measurement")
    p.add_argument("--serve-requests", type=int, default=1000)
    p.add_argument("--c1-stripes", type=int, default=64, help="stripes of the 64 MiB-shard leg")
    p.add_argument("--case", default=None, choices=sorted(CASES),
                   help="run one kernel family on one small case (for profiling) instead of the benchmark")
    p.add_argument("--case-mib", type=float, default=4.0, help="shard / buffer MiB of --case")
    p.add_argument("--kernel", default="auto", choices=["auto", "nibble", "byte", "gf2mma"],
                   help="kernel family for --case (where the shape allows it)")
    return p.parse_args()


def erasure_patterns(nst: int, seed: int = 0x5EED):
    rng = np.random.default_rng(seed)
    return [tuple(sorted(rng.choice(N_ALL, size=M_PAR, replace=False).tolist())) for _ in range(nst)]


def rank_seeds(rank: int) -> tuple[int, int]:
    """Seeds of a rank's own stripes (data, erasure patterns): under torchrun
    every rank encodes and rebuilds its own batch (weak scaling)."""
    return 0x1234 + rank, 0x5EED + rank


def max_over_ranks(ms: float, dist=None, device=None) -> float:
    """The slowest rank's time: the job ends when its last rank does."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_source_gbps(src_bytes_per_rank_step: int, world: int, ms_per_step: float) -> float:
    """Whole-job source GB/s: every rank's bytes over the slowest rank's time."""
    return src_bytes_per_rank_step * world / (ms_per_step / 1e3) / 1e9


def config(args, L):
    return {
        "workload": f"RS(10,4) Gf8D, {args.stripes} stripes x {L >> 10} KiB shards: batched encode "
                    f"(dot_product_matrix_with) + rebuild of 4 seeded erasures per stripe in place "
                    f"(mul_add_matrix_scattered semantics into zeroed rows, fused as "
                    f"dot_product_matrix_scattered_with; cached decode plans)",
        "field": "Gf8D (0x11D)", "k": K_SRC, "m": M_PAR, "stripes_per_gpu": args.stripes,
        "shard_bytes": L, "matrix": "Cauchy inv(x_i + y_j), x_i = 10 + i, y_j = j",
        "l2": "inputs (%.1f GiB per GPU) larger than L2 (126 MB)" % (args.stripes * N_ALL * L / 2 ** 30),
        "parallelism": f"replicas x{args.gpus} (stripes sharded across ranks, no collective)",
    }


# ---------------------------------------------------------------- CPU baseline (oracle port)

class PortJob(C.Structure):
    _fields_ = [("field", C.c_int), ("k", C.c_size_t), ("m", C.c_size_t), ("row_len", C.c_size_t),
                ("coeffs", C.c_void_p), ("srcs", C.c_void_p), ("rows", C.c_void_p), ("overwrite", C.c_int)]


def _port_lib():
    from oracle import orc

    lib = orc.L()
    lib.orc_port_supported.restype = C.c_int
    return lib if lib.orc_port_supported() else None


def cpu_baseline(L: int, seconds: float, nstripes: int = 16, threads: int | None = None):
    """Times the C restatement of the reference's AVX2+GFNI blocked kernels
    (oracle/cpu_port.c) on a bounded sample of the same workload (encode,
    then the rebuild of 4 erased shards written over), one stripe per job,
    on `threads` host threads (default: all)."""
    from oracle import orc
    from fgf_b200 import fields

    lib = _port_lib()
    if lib is None:
        return None
    cores = threads or os.cpu_count() or 1
    gf = fields.Gf8D
    cm = fields.cauchy(gf, M_PAR, K_SRC)
    enc = np.array(fields.encode_plan_coeffs(cm)[2], dtype=np.uint32)
    pats = erasure_patterns(nstripes, seed=0xC0DE)
    keep, jobs = [enc], []
    for s in range(nstripes):
        code = [orc.noise(L, 1000 * s + r) for r in range(N_ALL)]
        keep.append(code)
        sp = (C.c_void_p * K_SRC)(*[code[t].ctypes.data for t in range(K_SRC)])
        rp = (C.c_void_p * M_PAR)(*[code[K_SRC + j].ctypes.data for j in range(M_PAR)])
        keep += [sp, rp]
        jobs.append(PortJob(1, K_SRC, M_PAR, L, enc.ctypes.data, C.cast(sp, C.c_void_p),
                            C.cast(rp, C.c_void_p), 1))
        er = list(pats[s])
        sv = [i for i in range(N_ALL) if i not in er][:K_SRC]
        dm = fields.decode_rows(gf, cm, sv, er)
        dco = np.array([dm[j][t] for t in range(K_SRC) for j in range(M_PAR)], dtype=np.uint32)
        sp2 = (C.c_void_p * K_SRC)(*[code[i].ctypes.data for i in sv])
        rp2 = (C.c_void_p * M_PAR)(*[code[e].ctypes.data for e in er])
        keep += [dco, sp2, rp2]
        jobs.append(PortJob(1, K_SRC, M_PAR, L, dco.ctypes.data, C.cast(sp2, C.c_void_p),
                            C.cast(rp2, C.c_void_p), 1))
    arr = (PortJob * len(jobs))(*jobs)
    lib.orc_port_run_jobs(arr, C.c_size_t(len(jobs)), cores)  # warm-up (page faults)
    reps, t0 = 0, time.perf_counter()
    while True:
        lib.orc_port_run_jobs(arr, C.c_size_t(len(jobs)), cores)
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    src_bytes = reps * nstripes * 2 * K_SRC * L
    return {"value": round(src_bytes / el / 1e9, 2), "unit": "GB/s", "cores": cores, "kind": "port",
            "sample": f"{nstripes} stripes x RS(10,4) x {L >> 10} KiB encode+reconstruct, repeated {reps}x "
                      f"for {el:.1f} s on {cores} threads (oracle/cpu_port.c: AVX2+GFNI restatement of "
                      f"the reference's blocked kernels; the reference is Rust and not buildable here)"}


def cpu_one_core_64k(seconds: float):
    """One core, the config-0 shape the reference publishes (10 x 64 KiB ->
    4 parity rows, dot_product_matrix, 917,504 B working set: cache
    resident), for comparison with its single-core GiB/s figure."""
    from oracle import orc
    from fgf_b200 import fields

    lib = _port_lib()
    if lib is None:
        return None
    L = 64 << 10
    cm = fields.cauchy(fields.Gf8D, M_PAR, K_SRC)
    enc = np.array(fields.encode_plan_coeffs(cm)[2], dtype=np.uint32)
    code = [orc.noise(L, 77 + r) for r in range(N_ALL)]
    sp = (C.c_void_p * K_SRC)(*[code[t].ctypes.data for t in range(K_SRC)])
    rp = (C.c_void_p * M_PAR)(*[code[K_SRC + j].ctypes.data for j in range(M_PAR)])
    arr = (PortJob * 64)(*[PortJob(1, K_SRC, M_PAR, L, enc.ctypes.data, C.cast(sp, C.c_void_p),
                                   C.cast(rp, C.c_void_p), 1)] * 64)
    lib.orc_port_run_jobs(arr, C.c_size_t(64), 1)
    reps, t0 = 0, time.perf_counter()
    while True:
        lib.orc_port_run_jobs(arr, C.c_size_t(64), 1)
        reps += 1
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    b = reps * 64 * K_SRC * L
    return {"value_GiBps": round(b / el / 2 ** 30, 2), "value_GBps": round(b / el / 1e9, 2), "cores": 1,
            "kind": "port", "sample": f"RS(10,4) Gf8D encode of one 10 x 64 KiB stripe, {reps * 64} calls in "
                                      f"{el:.1f} s on 1 thread",
            "reference_published": "38.8-39.3 GiB/s, 1 core of a 4.8 GHz Core Ultra 7 258V "
                                   "(BENCHMARKS.md:260)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    L = int(args.shard_mib * 2 ** 20)
    per = max(1.0, args.cpu_seconds / max(1, args.steps))
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(L, per if i >= args.warmup else 0.5)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": "host CPU lacks AVX2+GFNI"}))
            return 0
        if i >= args.warmup:
            vals.append(r)
    v = float(np.median([x["value"] for x in vals]))
    base = dict(vals[-1])
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded LCG bytes)",
            "config": config(args, L), "cpu_baseline": base,
            "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- GPU arm: helpers

class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = [[x.strip() for x in r.split(",")] for r in out.strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [v for v in (num(r[1]) for r in rows) if v is not None]
        mx = [v for v in (num(r[2]) for r in rows) if v is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


class NvmlClockSampler:
    """SM clock and clock-event reasons read through NVML every ~2 ms during
    the timed region (reading only; nothing is set). The nvidia-smi loop
    above starts too slowly to sample a region of a few tens of ms."""

    def __init__(self, dev):
        import threading

        import pynvml as nv
        import torch

        self.nv = nv
        nv.nvmlInit()
        pr = torch.cuda.get_device_properties(dev)
        bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        self.h = nv.nvmlDeviceGetHandleByPciBusId(bus)
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM))
        self.rows = []
        self.stop_ev = threading.Event()
        self.first = threading.Event()
        self.thread = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        nv = self.nv
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        while not self.stop_ev.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.rows.append((mhz, sorted(n for n, b in bits.items() if rs & b)))
            except Exception:
                pass
            self.first.set()
            time.sleep(0.002)

    def start(self):
        self.thread.start()
        self.first.wait(timeout=2.0)

    def stop(self):
        self.stop_ev.set()
        self.thread.join(timeout=2.0)
        try:
            self.nv.nvmlShutdown()
        except Exception:
            pass
        if not self.rows:
            return None
        reasons = sorted({r for _, rs in self.rows for r in rs})
        return {"sm_mhz": float(np.median([m for m, _ in self.rows])), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.rows), "source": "nvml, every ~2 ms"}


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic():
    """DRAM bytes per step of the dominant kernels from the committed ncu
    summary (profiles/traffic.txt, `key: bytes` lines), or None."""
    p = ROOT / "profiles" / "traffic.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("rs104_batch_bytes_per_step:"):
            return float(line.split(":", 1)[1])
    return None


def event_ms(fn, reps: int, stream, warm: int = 3) -> float:
    """Mean milliseconds per call of `fn` on `stream`, CUDA events."""
    import torch

    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def windows(n: int, rng, count: int = 2, win: int = 4096) -> list[tuple[int, int]]:
    """16-byte-aligned column windows of an n-byte row: both ends and `count` inside."""
    out = [(0, min(win, n)), (max(0, n - win) // 16 * 16, n)]
    for _ in range(count):
        a = int(rng.integers(0, max(1, n - win))) // 16 * 16
        out.append((a, min(n, a + win)))
    return out


def oracle_matrix_windows(field_id: int, srcs, rows_before, rows_after, coeffs, overwrite: bool, rng) -> bool:
    """Every op of the family is independent column by column: the oracle on
    column windows of the sources gives the same windows of the rows. `srcs`
    and rows are device tensors (one per source / row)."""
    from oracle import orc

    n = srcs[0].numel()
    m = len(rows_after)
    for a, b in windows(n, rng):
        hs = [s[a:b].cpu().numpy().copy() for s in srcs]
        want = np.zeros(m * (b - a), np.uint8) if overwrite else \
            np.concatenate([r[a:b].cpu().numpy() for r in rows_before])
        (orc.dot_product_matrix if overwrite else orc.mul_add_matrix)(field_id, want, b - a, m, coeffs, hs)
        got = np.concatenate([r[a:b].cpu().numpy() for r in rows_after])
        if not np.array_equal(got, want):
            return False
    return True


# ---------------------------------------------------------------- mixed geometry

def mixed_geometry(n: int, seed: int, element_sizes=(1, 2)):
    """n stripe geometries: field Gf8D or Gf16 (50/50), k in U[4,32], m in
    U[1,8], shard length log-uniform in [4 KiB, 4 MiB] rounded down to the
    element size."""
    from fgf_b200.fields import Gf8D, Gf16

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        field = Gf8D if rng.random() < 0.5 else Gf16
        k = int(rng.integers(4, 33))
        m = int(rng.integers(1, 9))
        L = int(np.exp(rng.uniform(np.log(4096), np.log(4 << 20))))
        L -= L % field.BYTES
        out.append((field, k, m, L))
    return out


def uneven_batch(dev, nstripes: int, reps: int, tune_tiles: bool = False):
    """4096 stripes of mixed field / k / m / length, device-resident: one
    batched submission (work-list kernels, replayed as a CUDA graph) against
    the same stripes issued one call per stripe from a native loop. Each
    stripe's k sources are separate 256-byte-aligned shards; its m parity rows
    are contiguous (row j at j * L, as dot_product_matrix lays them out).
    Every 64th stripe is checked against the oracle on column windows before
    timing, and the two paths must agree on every byte."""
    import torch

    from fgf_b200 import batch as fb
    from fgf_b200 import ops
    from fgf_b200.fields import cauchy, encode_plan_coeffs

    geo = mixed_geometry(nstripes, 0xC3)
    up = lambda x: (x + 255) // 256 * 256
    src_total = sum(k * up(L) for _, k, _, L in geo)
    par_total = sum(up(m * L) for _, _, m, L in geo)
    pool = torch.empty(src_total, dtype=torch.uint8, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(0xC3C3)
    pool.random_(0, 256, generator=g)
    par_a = torch.zeros(par_total, dtype=torch.uint8, device=dev)
    par_b = torch.zeros(par_total, dtype=torch.uint8, device=dev)
    plans, coeffs_of = {}, {}
    jobs_a, jobs_b, views = [], [], []
    so = po = 0
    src_bytes = alg_bytes = 0
    for field, k, m, L in geo:
        key = (field.ID, k, m)
        if key not in plans:
            vals = encode_plan_coeffs(cauchy(field, m, k))[2]
            plans[key] = ops.Plan.matrix(field, k, m, vals)
            coeffs_of[key] = vals
        srcs = []
        for _ in range(k):
            srcs.append(pool[so:so + L])
            so += up(L)
        jobs_a.append(fb.Job(plans[key], srcs, par_a[po:po + m * L], L, m, True))
        jobs_b.append(fb.Job(plans[key], srcs, par_b[po:po + m * L], L, m, True))
        views.append((field, key, srcs, [par_a[po + j * L:po + (j + 1) * L] for j in range(m)]))
        po += up(m * L)
        src_bytes += k * L
        alg_bytes += (k + m) * L
    bt = fb.Batch(graphs=True)
    pa, pb = bt.prepare(jobs_a), bt.prepare(jobs_b)
    stream = torch.cuda.current_stream(dev)

    bt.run_prepared(pa, stream)
    torch.cuda.synchronize()
    rng = np.random.default_rng(0xC35)
    checked = list(range(0, nstripes, 64))
    oracle_ok = all(oracle_matrix_windows(views[i][0].ID, views[i][2], None, views[i][3], coeffs_of[views[i][1]],
                                          True, rng) for i in checked)

    ms_batched = event_ms(lambda: bt.run_prepared(pa, stream), reps, stream, warm=2)
    launches = bt.stats()["launches"]
    ms_plain = event_ms(lambda: fb.run_serial(pb, stream), reps, stream, warm=2)
    same = bool(torch.equal(par_a, par_b))
    # work-list tile shapes tuned on the first quarter of the stripes (every
    # class occurs there), then the whole batch again with the chosen tiles
    from fgf_b200 import tune
    tuned = {}
    if tune_tiles:
        sub = bt.prepare(jobs_a[:max(1, nstripes // 4)])
        t_before, t_after = tune.tune_batch_tiles(bt, sub, stream)
        ms_tuned = event_ms(lambda: bt.run_prepared(pa, stream), reps, stream, warm=2)
        torch.cuda.synchronize()
        tuned = {"tiles": {f"E{e}G{g}": tune.tile(e, g) for e in (1, 2, 4) for g in (1, 2, 3, 4)
                           if tune.tile(e, g) != 8},
                 "tuning_sample_us": [round(t_before, 1), round(t_after, 1)],
                 "ms": round(ms_tuned, 3), "source_GB/s": round(src_bytes / ms_tuned / 1e6, 1),
                 "hbm_frac": round(alg_bytes / ms_tuned / 1e6 / hbm_peak()[0], 4),
                 "vs_builtin_tiles": round(ms_batched / ms_tuned, 3),
                 "bit_identical": bool(torch.equal(par_a, par_b))}
    return {
        "workload": f"{nstripes} stripes, Gf8D/Gf16 50/50, k in [4,32], m in [1,8], shard length log-uniform "
                    f"4 KiB-4 MiB, Cauchy x_i = k + i, y_j = j; dot_product_matrix_with (encode)",
        "source_GB": round(src_bytes / 1e9, 2), "parity_GB": round((alg_bytes - src_bytes) / 1e9, 2),
        "batched": {"ms": round(ms_batched, 3), "source_GB/s": round(src_bytes / ms_batched / 1e6, 1),
                    "launches_per_pass": launches, "graph_replay": True},
        "one_call_per_stripe": {"ms": round(ms_plain, 3), "source_GB/s": round(src_bytes / ms_plain / 1e6, 1)},
        "speedup": round(ms_plain / ms_batched, 2),
        "bit_identical": same,
        "oracle_sample": {"stripes_checked": len(checked), "windows_per_stripe": 4, "passed": bool(oracle_ok)},
        "distinct_plans": len(plans),
        "hbm_frac_batched": round(alg_bytes / ms_batched / 1e6 / hbm_peak()[0], 4),
        "tuned_tiles": tuned,
    }


def served(dev, where: str, nreq: int, seconds_per_load: float):
    """Serving loop: Poisson arrivals of encode (70%) and reconstruct (30%)
    requests with mixed geometry, 20 coefficient matrices cached on the
    device, 64 GiB HBM budget. `where` = "host": shards in page-locked host
    memory (copied in and out); "device": shards already in HBM (in place).
    Saturation throughput first (all requests queued at once), then offered
    loads of 25-100% of it; each against the same requests served one at a
    time through the per-call entry points."""
    import torch

    from fgf_b200 import serve
    from fgf_b200.fields import cauchy, decode_rows, encode_plan_coeffs

    rng = np.random.default_rng(0xC4)
    geo = mixed_geometry(14, 0xC4)
    mats = []  # (field, k, m, coeffs, kind, row_starts_fn)
    for field, k, m, _ in geo:
        mats.append((field, k, m, encode_plan_coeffs(cauchy(field, m, k))[2], "encode", None))
    for field, k, m, _ in geo[:6]:
        cm = cauchy(field, m, k)
        er = sorted(rng.choice(k + m, size=m, replace=False).tolist())
        sv = [i for i in range(k + m) if i not in er][:k]
        dm = decode_rows(field, cm, sv, er)
        mats.append((field, k, len(er), [dm[j][t] for t in range(k) for j in range(len(er))], "reconstruct", er))
    maxL = 4 << 20
    if where == "host":
        src_pool = torch.empty(64 * maxL + 4096, dtype=torch.uint8).pin_memory()
        src_pool.random_(0, 256)
        ring = torch.empty(3 << 30, dtype=torch.uint8).pin_memory()
    else:
        src_pool = torch.empty(64 * maxL + 4096, dtype=torch.uint8, device=dev)
        src_pool.random_(0, 256)
        ring = torch.empty(3 << 30, dtype=torch.uint8, device=dev)
    ring_n = ring.numel()

    lens = mixed_geometry(nreq, 0xC44)
    reqs = []
    for i in range(nreq):
        enc = rng.random() < 0.7
        mi = int(rng.integers(0, 14)) if enc else 14 + int(rng.integers(0, 6))
        field, k, m, coeffs, kind, er = mats[mi]
        L = lens[i][3]
        L -= L % field.BYTES
        L = max(L, field.BYTES)
        offs = rng.integers(0, (64 * maxL - L) // 256, size=k) * 256  # shards start 256-byte aligned
        srcs = [src_pool[int(o):int(o) + L] for o in offs]
        if kind == "encode":
            need, starts = m * L, None
        else:
            need, starts = (k + m) * L, [e * L for e in er]
        pr = serve.PreparedRequest(field, coeffs, srcs, ring[:need], L, m, overwrite=kind == "encode",
                                   row_starts=starts)
        reqs.append((pr, need, (field, coeffs, srcs, L, m, kind, starts)))
    ring_addr = ring.data_ptr()

    def oracle_sample(srv, count: int = 24) -> dict:
        """Submit a sample of small requests together (so they share
        launches), then compare each destination with the oracle: encode
        overwrites its rows, reconstruct accumulates into scattered rows."""
        from oracle import orc

        pick = [i for i, (_, _, meta) in enumerate(reqs) if meta[3] <= (128 << 10)][:count]
        head, placed = 0, []
        fill = np.random.default_rng(0xC4C4)
        for i in pick:
            pr, need, meta = reqs[i]
            region = ring[head:head + need]
            before = fill.integers(0, 256, size=need, dtype=np.uint8)
            region.copy_(torch.from_numpy(before))
            pr.struct.dst = ring_addr + head
            placed.append((i, head, need, before))
            head += (need + 255) // 256 * 256
        torch.cuda.synchronize()
        tickets = [srv.submit_prepared(reqs[i][0]) for i, _, _, _ in placed]
        for t in tickets:
            srv.wait(t)
        bad = 0
        for i, h, need, before in placed:
            field, coeffs, srcs, L, m, kind, starts = reqs[i][2]
            got = ring[h:h + need].cpu().numpy()
            hs = [x.cpu().numpy().copy() for x in srcs]
            want = before.copy()
            if kind == "encode":
                orc.dot_product_matrix(field.ID, want, L, m, coeffs, hs)
            else:
                orc.mul_add_matrix_scattered(field.ID, want, L, starts, coeffs, hs)
            bad += 0 if np.array_equal(got, want) else 1
        srv.stats(reset=True)
        return {"requests_checked": len(placed), "mismatches": bad, "passed": bad == 0}

    def run(srv, rate: float | None, count: int):
        """Submit `count` requests (Poisson at `rate` per second, or all at
        once) with destinations carved from a ring; returns server stats."""
        srv.stats(reset=True)
        live = []  # (ticket, ring_start, ring_end), oldest first
        head = 0
        arr = np.random.default_rng(7).exponential(1.0 / rate, size=count) if rate else None
        t_next = time.perf_counter()
        for i in range(count):
            pr, need, _ = reqs[i % len(reqs)]
            if head + need > ring_n:
                head = 0
            while live and any(head < b1 and head + need > b0 for _, b0, b1 in live):
                srv.wait(live.pop(0)[0])
            if rate:
                t_next += arr[i]
                while time.perf_counter() < t_next:
                    pass
            pr.struct.dst = ring_addr + head  # the request is copied at submit; only the host data must wait
            t = srv.submit_prepared(pr)
            live.append((t, head, head + need))
            head += (need + 255) // 256 * 256
            while live and srv.poll(live[0][0]):
                live.pop(0)
        srv.drain()
        for t, _, _ in live:
            srv.wait(t)
        return srv.stats(reset=True)

    def summary(st):
        gbps = st["source_bytes"] / st["busy_s"] / 1e9 if st["busy_s"] else None
        return {"source_GB/s": round(gbps, 2) if gbps else None, "p50_us": round(st["p50_us"], 1),
                "p99_us": round(st["p99_us"], 1), "requests": st["completed"], "launches": st["launches"],
                "max_batch": st["max_batch_seen"], "plan_hits": st["plan_hits"], "plan_misses": st["plan_misses"],
                "peak_device_GB": round(st["peak_device_bytes"] / 1e9, 2),
                "queue_us": round(st["queue_us"], 1), "launch_us": round(st["launch_us"], 1)}

    srv_b = serve.Server(hbm_budget=64 << 30, staging_bytes=1 << 30)
    srv_p = serve.Server(hbm_budget=1 << 30, staging_bytes=1 << 30, plain=True)  # one request at a time
    try:
        checked = oracle_sample(srv_b)
        run(srv_b, None, min(64, nreq))  # warm-up: plans cached, kernels loaded
        run(srv_p, None, min(64, nreq))
        sat = run(srv_b, None, nreq)
        sat_plain = run(srv_p, None, nreq)
        rps = sat["completed"] / sat["busy_s"]
        mean_src = sat["source_bytes"] / max(1, sat["completed"])
        loads = []
        for frac in (0.25, 0.5, 0.75, 1.0):
            rate = frac * rps
            count = int(min(nreq, max(50, rate * seconds_per_load)))
            b = run(srv_b, rate, count)
            p = run(srv_p, rate, count)
            loads.append({"offered": frac, "requests_per_s": round(rate, 1), "requests": count,
                          "batched": summary(b), "plain": summary(p)})
    finally:
        srv_b.close()
        srv_p.close()
    return {
        "workload": f"{nreq} requests: 70% encode (dot_product_matrix) / 30% reconstruct "
                    f"(mul_add_matrix_scattered), geometry as the uneven batch, 20 device-cached matrices, "
                    + ("page-locked host shards copied in and out" if where == "host" else
                       "shards already in device memory (served in place)")
                    + f", HBM budget 64 GiB; mean {mean_src / 1e6:.1f} MB source per request",
        "saturation": {"batched": summary(sat), "plain": summary(sat_plain),
                       "speedup": round((sat["source_bytes"] / sat["busy_s"]) /
                                        (sat_plain["source_bytes"] / sat_plain["busy_s"]), 2)},
        "loads": loads,
        "oracle_sample": checked,
    }




# ---------------------------------------------------------------- other configurations

def leg_single_stripe(dev):
    """Config-0 shape as one call: RS(10,4) Gf8D encode of one stripe of
    10 x 64 KiB shards (917,504 B, L2-resident), dot_product_matrix_with,
    back-to-back calls: launch- and latency-bound."""
    import torch

    from fgf_b200 import ops
    from fgf_b200.fields import Gf8D, cauchy, encode_plan_coeffs
    from oracle import orc

    L = 64 << 10
    vals = encode_plan_coeffs(cauchy(Gf8D, M_PAR, K_SRC))[2]
    plan = ops.Plan.matrix(Gf8D, K_SRC, M_PAR, vals)
    code = torch.empty(N_ALL * L, dtype=torch.uint8, device=dev)
    data = [orc.noise(L, 0x5A + t) for t in range(K_SRC)]
    for t in range(K_SRC):
        code[t * L:(t + 1) * L] = torch.from_numpy(data[t]).to(dev)
    srcs = [code[t * L:(t + 1) * L] for t in range(K_SRC)]
    stream = torch.cuda.current_stream(dev)
    ops.dot_product_matrix_with(code[K_SRC * L:], L, M_PAR, plan, srcs, stream)
    torch.cuda.synchronize()
    want = np.zeros(M_PAR * L, np.uint8)
    orc.dot_product_matrix(Gf8D.ID, want, L, M_PAR, vals, data)
    ok = bool(np.array_equal(code[K_SRC * L:].cpu().numpy(), want))
    ms = event_ms(lambda: ops.dot_product_matrix_with(code[K_SRC * L:], L, M_PAR, plan, srcs, stream), 500, stream)
    # the same calls recorded once into a CUDA graph (100 calls) and replayed:
    # the device-side cost of a call without the Python binding's per-call
    # host work, which bounds the back-to-back figure above
    graph = None
    try:
        side = torch.cuda.Stream(dev)
        side.wait_stream(stream)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            cs = torch.cuda.current_stream(dev)
            for _ in range(100):
                ops.dot_product_matrix_with(code[K_SRC * L:], L, M_PAR, plan, srcs, cs)
        stream.wait_stream(side)
        code[K_SRC * L:].fill_(0)
        g.replay()
        torch.cuda.synchronize()
        gok = bool(np.array_equal(code[K_SRC * L:].cpu().numpy(), want))
        gms = event_ms(lambda: g.replay(), 20, stream) / 100
        graph = {"us_per_call": round(gms * 1e3, 2), "source_GiB/s": round(K_SRC * L / gms * 1e3 / 2 ** 30, 2),
                 "calls_per_graph": 100, "oracle": "passed" if gok else "FAILED"}
        del g
    except Exception as exc:  # capture refused: report why
        graph = {"unavailable": str(exc)[:200]}
    return {"workload": "RS(10,4) Gf8D encode, one stripe of 10 x 64 KiB (config 0), dot_product_matrix_with per "
                        "call, 500 calls back to back", "us_per_call": round(ms * 1e3, 2),
            "source_GB/s": round(K_SRC * L / ms / 1e6, 2), "source_GiB/s": round(K_SRC * L / ms * 1e3 / 2 ** 30, 2),
            "l2": "resident (917,504 B)", "oracle": "passed" if ok else "FAILED", "graph_replay": graph}


def leg_64mib(dev, nst: int, steps: int = 3):
    """Config-1 shape at 64 MiB shards: the headline step (batched encode +
    in-place rebuild of 4 erasures per stripe) on nst stripes; the 256-stripe
    batch would need 224 GiB, more than one GPU holds."""
    import torch

    from fgf_b200 import batch as fb
    from fgf_b200 import ops
    from fgf_b200.fields import Gf8D, cauchy, decode_rows, encode_plan_coeffs

    L = 64 * MIB
    stripe = N_ALL * L
    code = torch.empty(nst * stripe, dtype=torch.uint8, device=dev)
    g = torch.Generator(device=dev)
    g.manual_seed(0x64)
    code.random_(0, 256, generator=g)
    cm = cauchy(Gf8D, M_PAR, K_SRC)
    enc_plan = ops.Plan.matrix(Gf8D, *encode_plan_coeffs(cm))
    pats = erasure_patterns(nst, seed=0x64)
    cache = {}
    row = lambda s, r: code[s * stripe + r * L: s * stripe + (r + 1) * L]
    enc_jobs, rec_jobs = [], []
    for s in range(nst):
        enc_jobs.append(fb.Job(enc_plan, [row(s, t) for t in range(K_SRC)],
                               code[s * stripe + K_SRC * L:(s + 1) * stripe], L, M_PAR, True))
        er = pats[s]
        if er not in cache:
            sv = [i for i in range(N_ALL) if i not in er][:K_SRC]
            dm = decode_rows(Gf8D, cm, sv, list(er))
            cache[er] = (ops.Plan.matrix(Gf8D, K_SRC, M_PAR, [dm[j][t] for t in range(K_SRC) for j in range(M_PAR)]), sv)
        plan, sv = cache[er]
        rec_jobs.append(fb.Job(plan, [row(s, i) for i in sv], code[s * stripe:(s + 1) * stripe], L, M_PAR, True,
                               [e * L for e in er]))
    bt = fb.Batch(graphs=True)
    pe, pr = bt.prepare(enc_jobs), bt.prepare(rec_jobs)
    stream = torch.cuda.current_stream(dev)
    bt.run_prepared(pe, stream)
    torch.cuda.synchronize()
    check = [0, nst - 1]
    truth = {s: [row(s, e).clone() for e in pats[s]] for s in check}
    for s in check:
        for e in pats[s]:
            row(s, e).fill_(0xEE)  # erased rows hold garbage; the rebuild overwrites them
    bt.run_prepared(pr, stream)
    torch.cuda.synchronize()
    ok = all(torch.equal(row(s, e), truth[s][j]) for s in check for j, e in enumerate(pats[s]))
    del truth
    enc_ms = event_ms(lambda: bt.run_prepared(pe, stream), steps, stream, warm=1)
    rec_ms = event_ms(lambda: bt.run_prepared(pr, stream), steps, stream, warm=1)
    peak = hbm_peak()[0]
    alg = nst * 2 * N_ALL * L
    ms = enc_ms + rec_ms
    return {"workload": f"RS(10,4) Gf8D, {nst} stripes x 64 MiB shards ({nst * stripe / 2 ** 30:.0f} GiB; 256 "
                        f"stripes would need 224 GiB): batched encode + in-place rebuild of 4 erasures",
            "ms_per_step": round(ms, 3), "source_GB/s": round(nst * 2 * K_SRC * L / ms / 1e6, 1),
            "hbm_frac": round(alg / ms / 1e6 / peak, 4), "encode_ms": round(enc_ms, 3),
            "rebuild_ms": round(rec_ms, 3), "rebuilt_bit_exact": bool(ok)}


def leg_single_row_ops(dev):
    """Config-1 single-row ops on 256 MiB buffers with random nonzero
    coefficients: mul_add (3 L bytes), mul_add_scatter 1 -> 4 ((1 + 2*4) L),
    mul_add_gather 4 -> 1 ((4 + 2) L). Checked on windows against the oracle."""
    import torch

    from fgf_b200 import ops
    from fgf_b200.fields import Gf8D
    from oracle import orc

    n = 256 * MIB
    rng = np.random.default_rng(0x256)
    g = torch.Generator(device=dev)
    g.manual_seed(0x256)
    c = [int(x) for x in rng.integers(1, 256, size=4)]
    src = torch.randint(0, 256, (n,), dtype=torch.uint8, device=dev, generator=g)
    rows = torch.randint(0, 256, (4 * n,), dtype=torch.uint8, device=dev, generator=g)
    dst = torch.randint(0, 256, (n,), dtype=torch.uint8, device=dev, generator=g)
    stream = torch.cuda.current_stream(dev)
    peak = hbm_peak()[0]
    out = {}
    ok = True
    # parity first
    d0, r0 = dst.clone(), rows.clone()
    ops.mul_add(Gf8D, dst, c[0], src)
    ops.mul_add_scatter(Gf8D, rows, n, c, src)
    torch.cuda.synchronize()
    for a, b in windows(n, rng):
        hs = src[a:b].cpu().numpy().copy()
        w = d0[a:b].cpu().numpy().copy()
        orc.mul_add(Gf8D.ID, w, c[0], hs)
        ok &= bool(np.array_equal(dst[a:b].cpu().numpy(), w))
        for j in range(4):
            w = r0[j * n + a:j * n + b].cpu().numpy().copy()
            orc.mul_add(Gf8D.ID, w, c[j], hs)
            ok &= bool(np.array_equal(rows[j * n + a:j * n + b].cpu().numpy(), w))
    del d0, r0
    gsrcs = [rows[j * n:(j + 1) * n] for j in range(4)]
    d1 = dst.clone()
    ops.mul_add_gather(Gf8D, dst, c, gsrcs)
    torch.cuda.synchronize()
    for a, b in windows(n, rng):
        w = d1[a:b].cpu().numpy().copy()
        orc.mul_add_gather(Gf8D.ID, w, c, [s[a:b].cpu().numpy().copy() for s in gsrcs])
        ok &= bool(np.array_equal(dst[a:b].cpu().numpy(), w))
    del d1
    for name, fn, alg, srcb in (
            ("mul_add", lambda: ops.mul_add(Gf8D, dst, c[0], src, stream), 3 * n, n),
            ("mul_add_scatter_1to4", lambda: ops.mul_add_scatter(Gf8D, rows, n, c, src, stream), 9 * n, n),
            ("mul_add_gather_4to1", lambda: ops.mul_add_gather(Gf8D, dst, c, gsrcs, stream), 6 * n, 4 * n)):
        ms = event_ms(fn, 10, stream)
        out[name] = {"ms": round(ms, 4), "GB/s": round(alg / ms / 1e6, 1), "hbm_frac": round(alg / ms / 1e6 / peak, 4),
                     "source_GB/s": round(srcb / ms / 1e6, 1)}
    out["workload"] = "Gf8D, 256 MiB buffers, random nonzero coefficients (config 1 single-row ops)"
    out["oracle_windows"] = "passed" if ok else "FAILED"
    return out


def leg_tower_and_large_km(dev):
    """Config-2 shapes, dot_product_matrix_with with uniformly random nonzero
    coefficients: Gf16 RS(32,8) on 16 MiB shards, Gf32 RS(16,4) on 8 MiB,
    Gf8B RS(64,16) on 4 MiB. Each kernel variant the library offers for the
    shape is timed (the tuner's choice first), every variant checked against
    the oracle on column windows."""
    import torch

    from fgf_b200 import ops, tune
    from fgf_b200.fields import Gf8B, Gf16, Gf32

    peak = hbm_peak()[0]
    out = {}
    stream = torch.cuda.current_stream(dev)
    for name, field, k, m, L in (("gf16_rs32_8_16MiB", Gf16, 32, 8, 16 * MIB),
                                 ("gf32_rs16_4_8MiB", Gf32, 16, 4, 8 * MIB),
                                 ("gf8b_rs64_16_4MiB", Gf8B, 64, 16, 4 * MIB)):
        rng = np.random.default_rng(0xC2 + field.ID)
        g = torch.Generator(device=dev)
        g.manual_seed(0xC2 + field.ID)
        vals = [int(x) for x in rng.integers(1, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]
        plan = ops.Plan.matrix(field, k, m, vals)
        buf = torch.randint(0, 256, ((k + m) * L,), dtype=torch.uint8, device=dev, generator=g)
        srcs = [buf[t * L:(t + 1) * L] for t in range(k)]
        rows = buf[k * L:]
        rows_v = [rows[j * L:(j + 1) * L] for j in range(m)]
        res = {"k": k, "m": m, "shard_bytes": L}
        for variant in tune.variants_for(field, k, m, L):
            with tune.forced(variant):
                rows.fill_(0xA5)
                ops.dot_product_matrix_with(rows, L, m, plan, srcs, stream)
                torch.cuda.synchronize()
                ok = oracle_matrix_windows(field.ID, srcs, None, rows_v, vals, True, rng)
                ms = event_ms(lambda: ops.dot_product_matrix_with(rows, L, m, plan, srcs, stream), 10, stream)
            alg = (k + m) * L
            res[variant] = {"ms": round(ms, 4), "source_GB/s": round(k * L / ms / 1e6, 1),
                            "hbm_frac": round(alg / ms / 1e6 / peak, 4), "oracle_windows": "passed" if ok else "FAILED"}
        res["chosen"] = tune.chosen(field, k, m, L)
        out[name] = res
        del buf
        torch.cuda.empty_cache()
    return out


def leg_wide_fields(dev, L: int = 16 * MIB):
    """The 8-byte fields (GF(2^64), Fan-Paar GF(2^64)): RS(10,4) encode with
    dot_product_matrix_with on 16 MiB shards, uniformly random 64-bit
    coefficients, on the 8-byte table kernel; checked against the oracle on
    column windows."""
    import torch

    from fgf_b200 import ops
    from fgf_b200.fields import FanPaar64, Gf64

    peak = hbm_peak()[0]
    out = {}
    stream = torch.cuda.current_stream(dev)
    k, m = 10, 4
    for name, field in (("gf64_rs10_4_16MiB", Gf64), ("fp64_rs10_4_16MiB", FanPaar64)):
        rng = np.random.default_rng(0x64 + field.ID)
        g = torch.Generator(device=dev)
        g.manual_seed(0x64 + field.ID)
        vals = [int(x) for x in rng.integers(1, 1 << 64, size=k * m, dtype=np.uint64)]
        plan = ops.Plan.matrix(field, k, m, vals)
        buf = torch.randint(0, 256, ((k + m) * L,), dtype=torch.uint8, device=dev, generator=g)
        srcs = [buf[t * L:(t + 1) * L] for t in range(k)]
        rows = buf[k * L:]
        rows.fill_(0xA5)
        ops.dot_product_matrix_with(rows, L, m, plan, srcs, stream)
        torch.cuda.synchronize()
        ok = oracle_matrix_windows(field.ID, srcs, None, [rows[j * L:(j + 1) * L] for j in range(m)], vals, True, rng)
        ms = event_ms(lambda: ops.dot_product_matrix_with(rows, L, m, plan, srcs, stream), 10, stream)
        out[name] = {"ms": round(ms, 4), "source_GB/s": round(k * L / ms / 1e6, 1),
                     "hbm_frac": round((k + m) * L / ms / 1e6 / peak, 4), "oracle_windows": "passed" if ok else "FAILED"}
        del buf
        torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- GPU arm

def pcie_duplex(dev, nbytes: int = 1 << 30) -> dict:
    """Host<->device copy bandwidth with both directions busy at once
    (page-locked host memory, one stream per direction)."""
    import torch

    h_in = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    h_out = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d_in = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d_out = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    res = {}
    for _ in range(2):
        torch.cuda.synchronize()
        e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        e[0].record(s1)
        e[2].record(s2)
        with torch.cuda.stream(s1):
            d_in.copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s2):
            h_out.copy_(d_out, non_blocking=True)
        e[1].record(s1)
        e[3].record(s2)
        torch.cuda.synchronize()
        res = {"h2d_GB/s": round(nbytes / e[0].elapsed_time(e[1]) / 1e6, 1),
               "d2h_GB/s": round(nbytes / e[2].elapsed_time(e[3]) / 1e6, 1)}
    del h_in, h_out, d_in, d_out
    return res


def run_ours(args):
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from fgf_b200 import batch as fb
    from fgf_b200 import ops
    from fgf_b200.fields import Gf8D, cauchy, decode_rows, encode_plan_coeffs

    L = int(args.shard_mib * 2 ** 20)
    nst = args.stripes
    stripe = N_ALL * L
    code = torch.empty(nst * stripe, dtype=torch.uint8, device=dev)
    g = torch.Generator(device=dev)
    data_seed, pattern_seed = rank_seeds(rank)
    g.manual_seed(data_seed)
    code.random_(0, 256, generator=g)
    cm = cauchy(Gf8D, M_PAR, K_SRC)
    enc_plan = ops.Plan.matrix(Gf8D, *encode_plan_coeffs(cm))
    pats = erasure_patterns(nst, seed=pattern_seed)
    cache = {}

    def dec_plan(er):
        if er not in cache:
            sv = [i for i in range(N_ALL) if i not in er][:K_SRC]
            dm = decode_rows(Gf8D, cm, sv, list(er))
            cache[er] = (ops.Plan.matrix(Gf8D, K_SRC, M_PAR, [dm[j][t] for t in range(K_SRC)
                                                                for j in range(M_PAR)]), sv)
        return cache[er]

    def row(s, r):
        return code[s * stripe + r * L: s * stripe + (r + 1) * L]

    enc_jobs = [fb.Job(enc_plan, [row(s, t) for t in range(K_SRC)],
                       code[s * stripe + K_SRC * L: (s + 1) * stripe], L, M_PAR, True) for s in range(nst)]
    rec_jobs = []
    for s in range(nst):
        plan, sv = dec_plan(pats[s])
        rec_jobs.append(fb.Job(plan, [row(s, i) for i in sv], code[s * stripe:(s + 1) * stripe], L, M_PAR,
                               True, [e * L for e in pats[s]]))
    bt = fb.Batch(graphs=True)
    enc_p, rec_p = bt.prepare(enc_jobs), bt.prepare(rec_jobs)
    stream = torch.cuda.current_stream(dev)

    # ---- correctness of one step: encode vs oracle (stripe 0 whole, sampled
    # stripes on windows); erased shards filled with garbage are rebuilt
    # bit-exactly on sampled stripes
    bt.run_prepared(enc_p, stream)
    torch.cuda.synchronize()
    check = list(range(0, nst, max(1, nst // 8)))
    truth = {s: [row(s, e).cpu().numpy().copy() for e in pats[s]] for s in check}
    for s in range(nst):
        for e in pats[s]:
            row(s, e).fill_(0xEE)
    bt.run_prepared(rec_p, stream)
    torch.cuda.synchronize()
    ok = all(np.array_equal(row(s, e).cpu().numpy(), truth[s][j]) for s in check for j, e in enumerate(pats[s]))
    if rank == 0:
        from oracle import orc

        h0 = code[:stripe].cpu().numpy()
        want = np.zeros(M_PAR * L, np.uint8)
        vals = encode_plan_coeffs(cm)[2]
        orc.dot_product_matrix(1, want, L, M_PAR, vals, [h0[t * L:(t + 1) * L].copy() for t in range(K_SRC)])
        ok = ok and np.array_equal(h0[K_SRC * L:], want)
        rng = np.random.default_rng(0x0C)
        for s in check[1:]:
            ok = ok and oracle_matrix_windows(1, [row(s, t) for t in range(K_SRC)], None,
                                              [row(s, K_SRC + j) for j in range(M_PAR)], vals, True, rng)
    if not ok:
        print(json.dumps({"metric": METRIC, "error": "parity check failed"}))
        return 1

    # ---- timed region: W warm-up steps, K timed steps, events per submission
    for _ in range(args.warmup):
        bt.run_prepared(enc_p, stream)
        bt.run_prepared(rec_p, stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    try:
        sampler = NvmlClockSampler(dev)
    except Exception:  # no NVML: the nvidia-smi loop
        sampler = ClockSampler(local)
    sampler.start()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    launches = 0
    torch.cuda.synchronize()
    start.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        bt.run_prepared(enc_p, stream)
        launches += bt.stats()["launches"]
        ev[i][1].record(stream)
        bt.run_prepared(rec_p, stream)
        launches += bt.stats()["launches"]
        ev[i][2].record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = start.elapsed_time(end)
    enc_ms = sum(e[0].elapsed_time(e[1]) for e in ev) / args.steps
    rec_ms = sum(e[1].elapsed_time(e[2]) for e in ev) / args.steps
    if dist:
        ms = max_over_ranks(ms, dist, dev)
        dist.barrier()
    ms_step = ms / args.steps
    src_per_step = nst * 2 * K_SRC * L * world
    value = job_source_gbps(nst * 2 * K_SRC * L, world, ms_step)

    # ---- roofline of the dominant kernels (byte-table batch kernels, K = 10)
    peak, peak_kind = hbm_peak()
    enc_bytes = nst * (K_SRC + M_PAR) * L            # read 10, write 4
    rec_bytes = nst * (K_SRC + M_PAR) * L            # read 10 survivors, write 4 rebuilt rows
    achieved = (enc_bytes + rec_bytes) / ((enc_ms + rec_ms) / 1e3) / 1e9
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
            "traffic": profiled_traffic(), "algorithmic_bytes_per_step": enc_bytes + rec_bytes,
            "encode": {"ms": round(enc_ms, 4), "GB/s": round(enc_bytes / enc_ms / 1e6, 1),
                       "frac": round(enc_bytes / enc_ms / 1e6 / peak, 4),
                       "source_GB/s": round(nst * K_SRC * L / enc_ms / 1e6, 1),
                       "kernel": "batch_fast_uniform_kernel<10> (one plan for every stripe)"},
            "reconstruct": {"ms": round(rec_ms, 4), "GB/s": round(rec_bytes / rec_ms / 1e6, 1),
                            "frac": round(rec_bytes / rec_ms / 1e6 / peak, 4),
                            "source_GB/s": round(nst * K_SRC * L / rec_ms / 1e6, 1),
                            "kernel": "batch_fast_segment_kernel<10> (contiguous column range per CTA, per-stripe decode plans, overwrite)"},
            "note": "achieved = algorithmic bytes of both submissions / their CUDA-event time; the rebuild "
                    "overwrites the erased rows, so it reads 10 and writes 4 shards per stripe"}

    # ---- e2e: host buffers through the public API, copies inside the timed
    # region. Device layout: data shards [stripe][10 L], then per stripe the
    # 4 parity rows and the 4 rebuilt rows [stripe][8 L], so every chunk of
    # stripes goes in with one copy and its results come out with one copy.
    # Chunks run on three streams (copy in, compute, copy out), so copies of
    # neighbouring chunks overlap in both directions and the kernels hide
    # under them.
    e2e, pcie = None, None
    if not args.no_e2e:
        del code
        torch.cuda.empty_cache()
        pcie = pcie_duplex(dev)
        dsz, osz = K_SRC * L, 2 * M_PAR * L
        D = torch.empty(nst * (dsz + osz), dtype=torch.uint8, device=dev)
        D.random_(0, 256, generator=g)
        dbase = nst * dsz

        def shard(s, i):  # offset of shard i of stripe s
            return s * dsz + i * L if i < K_SRC else dbase + s * osz + (i - K_SRC) * L

        host_in = torch.empty(nst, dsz, dtype=torch.uint8).pin_memory()
        host_in.copy_(D[:dbase].view(nst, dsz).cpu())
        host_out = torch.empty(nst, osz, dtype=torch.uint8).pin_memory()
        per = max(1, min(nst, 16))
        chunks = [list(range(c, min(nst, c + per))) for c in range(0, nst, per)]
        ejobs, rjobs = [], []
        for s in range(nst):
            ejobs.append(fb.Job(enc_plan, [D[shard(s, t):shard(s, t) + L] for t in range(K_SRC)],
                                D[dbase + s * osz: dbase + s * osz + M_PAR * L], L, M_PAR, True))
            plan, sv = dec_plan(pats[s])
            rjobs.append(fb.Job(plan, [D[shard(s, i):shard(s, i) + L] for i in sv], D, L, M_PAR, True,
                                [dbase + s * osz + (M_PAR + j) * L for j in range(M_PAR)]))
        # one batch object per chunk: its descriptor slots are reused only by
        # the same chunk one step later, so issuing never waits on other chunks
        bt_c = [fb.Batch(graphs=True) for _ in chunks]
        enc_c = [bt_c[c].prepare([ejobs[s] for s in ch]) for c, ch in enumerate(chunks)]
        rec_c = [bt_c[c].prepare([rjobs[s] for s in ch]) for c, ch in enumerate(chunks)]
        s_in = torch.cuda.Stream(dev)
        s_out = torch.cuda.Stream(dev)
        ev_in = [torch.cuda.Event() for _ in chunks]
        ev_run = [torch.cuda.Event() for _ in chunks]
        ev_out = [torch.cuda.Event() for _ in chunks]
        for c in range(len(chunks)):  # recorded once so the first waits are no-ops
            ev_run[c].record(stream)
            ev_out[c].record(stream)
        copies = [0]

        def e2e_step():
            for c, ch in enumerate(chunks):
                a, b = ch[0], ch[-1] + 1
                s_in.wait_event(ev_run[c])      # the previous step's kernels are done with these shards
                with torch.cuda.stream(s_in):
                    D[a * dsz:b * dsz].view(b - a, dsz).copy_(host_in[a:b], non_blocking=True)
                ev_in[c].record(s_in)
                stream.wait_event(ev_in[c])
                stream.wait_event(ev_out[c])    # the previous step's results have left
                bt_c[c].run_prepared(enc_c[c], stream)
                bt_c[c].run_prepared(rec_c[c], stream)
                ev_run[c].record(stream)
                s_out.wait_event(ev_run[c])
                with torch.cuda.stream(s_out):
                    host_out[a:b].copy_(D[dbase + a * osz:dbase + b * osz].view(b - a, osz), non_blocking=True)
                ev_out[c].record(s_out)
                copies[0] += 2

        for _ in range(3):  # warm-up: every descriptor slot captures its graph
            e2e_step()
        torch.cuda.synchronize()
        # results in host memory: parity vs the oracle on column windows and
        # rebuilt shards vs the originals they replace, for the checked stripes
        from oracle import orc

        e2e_ok = True
        rng_e = np.random.default_rng(0xE2E)
        vals = encode_plan_coeffs(cm)[2]
        for s in check:
            for a, b in windows(L, rng_e):
                want = np.zeros(M_PAR * (b - a), np.uint8)
                orc.dot_product_matrix(1, want, b - a, M_PAR, vals,
                                       [host_in[s, t * L + a:t * L + b].numpy().copy() for t in range(K_SRC)])
                got = np.concatenate([host_out[s, j * L + a:j * L + b].numpy() for j in range(M_PAR)])
                e2e_ok &= bool(np.array_equal(got, want))
            for j, e in enumerate(pats[s]):
                orig = host_in[s, e * L:(e + 1) * L].numpy() if e < K_SRC else \
                    host_out[s, (e - K_SRC) * L:(e - K_SRC + 1) * L].numpy()
                e2e_ok &= bool(np.array_equal(host_out[s, (M_PAR + j) * L:(M_PAR + j + 1) * L].numpy(), orig))
        want_out = host_out.clone()
        es = max(1, min(args.steps, 5))
        if dist:
            dist.barrier()
        copies[0] = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s_in.wait_stream(stream)
        s_out.wait_stream(stream)
        for _ in range(es):
            e2e_step()
        stream.wait_stream(s_in)
        stream.wait_stream(s_out)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        same = bool(torch.equal(host_out, want_out))
        if dist:
            ems = max_over_ranks(ems, dist, dev)
        h2d, d2h = nst * dsz, nst * osz
        bound_ms = max(h2d / pcie["h2d_GB/s"], d2h / pcie["d2h_GB/s"]) / 1e6
        e2e = {"value": round(src_per_step / (ems / es / 1e3) / 1e9, 2), "unit": "GB/s",
               "h2d_bytes_per_step": h2d * world, "d2h_bytes_per_step": d2h * world,
               "steps": es, "chunks": len(chunks), "copies_per_step": copies[0] // es,
               "results_checked": e2e_ok, "results_repeatable": same,
               "pcie_duplex": pcie, "pcie_bound_ms": round(bound_ms, 2), "ms_per_step": round(ems / es, 2),
               "pcie_frac": round(bound_ms / (ems / es), 4),
               "note": "page-locked host data shards in, parity and rebuilt shards out, per step; one copy in "
                       "and one copy out per chunk of %d stripes, on their own streams" % per}
        del D, host_in, host_out, want_out
        torch.cuda.empty_cache()
        if not e2e_ok:
            print(json.dumps({"metric": METRIC, "error": "e2e results differ"}))
            return 1
    else:
        del code
        torch.cuda.empty_cache()

    extra, compact = {}, {}
    if world == 1 and not args.no_legs:
        legs = {"config0_single_stripe_64KiB": leg_single_stripe(dev)}
        torch.cuda.empty_cache()
        legs["config1_64MiB_shards"] = leg_64mib(dev, args.c1_stripes)
        torch.cuda.empty_cache()
        legs["config1_single_row_256MiB"] = leg_single_row_ops(dev)
        torch.cuda.empty_cache()
        legs["config2_tower_large_km"] = leg_tower_and_large_km(dev)
        legs["fields_64bit_rs10_4"] = leg_wide_fields(dev)
        torch.cuda.empty_cache()
        extra["legs"] = legs
        compact["c0_us_per_call"] = legs["config0_single_stripe_64KiB"]["us_per_call"]
        c0g = legs["config0_single_stripe_64KiB"]["graph_replay"] or {}
        if "us_per_call" in c0g:
            compact["c0_graph_us_per_call"] = c0g["us_per_call"]
        compact["c1_64MiB_source_GBps"] = legs["config1_64MiB_shards"]["source_GB/s"]
        compact["c1_64MiB_hbm_frac"] = legs["config1_64MiB_shards"]["hbm_frac"]
        for k_, v_ in legs["config1_single_row_256MiB"].items():
            if isinstance(v_, dict):
                compact[f"{k_}_256MiB_hbm_frac"] = v_["hbm_frac"]
        for k_, v_ in legs["config2_tower_large_km"].items():
            compact[f"c2_{k_}_source_GBps"] = v_[v_["chosen"]]["source_GB/s"]
            compact[f"c2_{k_}_kernel"] = v_["chosen"]
        for k_, v_ in legs["fields_64bit_rs10_4"].items():
            compact[f"{k_}_source_GBps"] = v_["source_GB/s"]
    if world == 1 and not args.no_uneven:
        u = uneven_batch(dev, args.uneven_stripes, 5, tune_tiles=True)
        extra["uneven_batch"] = u
        compact.update({"uneven_speedup": u["speedup"], "uneven_batched_source_GBps": u["batched"]["source_GB/s"],
                        "uneven_hbm_frac": u["hbm_frac_batched"], "uneven_oracle": u["oracle_sample"]["passed"]})
        if u["tuned_tiles"]:
            compact.update({"uneven_tuned_hbm_frac": u["tuned_tiles"]["hbm_frac"],
                            "uneven_tuned_vs_builtin_tiles": u["tuned_tiles"]["vs_builtin_tiles"]})
        torch.cuda.empty_cache()  # its buffers are free now; hand them back before the serving loop allocates
    if world == 1 and not args.no_serve:
        sv_host = served(dev, "host", args.serve_requests, 0.5)
        torch.cuda.empty_cache()
        sv_dev = served(dev, "device", 4 * args.serve_requests, 0.25)
        torch.cuda.empty_cache()
        extra["served"] = {"host": sv_host, "device": sv_dev}
        for w, sv in (("host", sv_host), ("device", sv_dev)):
            sat = sv["saturation"]
            compact[f"served_{w}_speedup"] = sat["speedup"]
            compact[f"served_{w}_source_GBps"] = sat["batched"]["source_GB/s"]
            compact[f"served_{w}_p50_us"] = sat["batched"]["p50_us"]
            compact[f"served_{w}_p99_us"] = sat["batched"]["p99_us"]
            compact[f"served_{w}_oracle"] = sv["oracle_sample"]["passed"]

    cpu, cpu1 = None, None
    if rank == 0 and not args.no_cpu and world == 1:
        cpu = cpu_baseline(L, args.cpu_seconds)
        cpu1 = cpu_one_core_64k(min(5.0, args.cpu_seconds))
        if cpu1:
            compact["cpu_1core_64KiB_GiBps"] = cpu1["value_GiBps"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    compact["encode_hbm_frac"] = roof["encode"]["frac"]
    compact["reconstruct_hbm_frac"] = roof["reconstruct"]["frac"]
    if e2e:
        compact["e2e_pcie_frac"] = e2e["pcie_frac"]
    line = {"metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded uniform random bytes; seeded erasure patterns)",
            "config": config(args, L), "roofline": roof, "cpu_baseline": cpu, "cpu_baseline_1core": cpu1,
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "parity_check": "passed",
            "value_GiBps": round(value * 1e9 / 2 ** 30, 2), **compact, **extra}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- single cases (profiling)

CASES = {
    # name: (field name, k, m) for dot_product_matrix_with, or an op name
    "c2_gf16": ("Gf16", 32, 8), "c2_gf32": ("Gf32", 16, 4), "c2_gf8b": ("Gf8B", 64, 16),
    "rs104_encode": ("Gf8D", 10, 4), "gf16_rs8_2": ("Gf16", 8, 2),
    "gf64_rs104": ("Gf64", 10, 4), "fp64_rs104": ("FanPaar64", 10, 4),
    "axpy": "mul_add", "scatter": "mul_add_scatter", "gather": "mul_add_gather",
    "xor": "add_assign", "elementwise": "mul_elementwise", "uneven": "uneven", "batch_gf16_12_8": "batch16",
}


def run_case(args):
    """One kernel family on one case: checked once against the oracle on
    column windows, then run --steps times back to back (CUDA events)."""
    import torch

    from fgf_b200 import fields, ops, tune
    from oracle import orc

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    n = int(args.case_mib * MIB)
    rng = np.random.default_rng(0xCA5E)
    g = torch.Generator(device=dev)
    g.manual_seed(0xCA5E)
    spec = CASES[args.case]
    tune.force(args.kernel)
    ok = True
    if isinstance(spec, tuple):
        field = getattr(fields, spec[0])
        k, m = spec[1], spec[2]
        n -= n % field.BYTES
        vals = [int(x) for x in rng.integers(1, 1 << (8 * field.BYTES), size=k * m, dtype=np.uint64)]
        plan = ops.Plan.matrix(field, k, m, vals)
        buf = torch.randint(0, 256, ((k + m) * n,), dtype=torch.uint8, device=dev, generator=g)
        srcs = [buf[t * n:(t + 1) * n] for t in range(k)]
        rows = buf[k * n:]
        fn = lambda: ops.dot_product_matrix_with(rows, n, m, plan, srcs, stream)
        fn()
        torch.cuda.synchronize()
        ok = oracle_matrix_windows(field.ID, srcs, None, [rows[j * n:(j + 1) * n] for j in range(m)], vals, True, rng)
        alg, src_b = (k + m) * n, k * n
        kernel = "wide" if field.BYTES == 8 else tune.chosen(field, k, m, n)
    elif spec == "batch16":
        # one batched submission of 64 Gf16 stripes, 12 sources and 8 rows of
        # case-mib MiB each, every stripe its own plan
        from fgf_b200 import batch as fb
        field, k, m, ns = fields.Gf16, 12, 8, 64
        n -= n % 2
        buf = torch.randint(0, 256, (ns * (k + m) * n,), dtype=torch.uint8, device=dev, generator=g)
        jobs, chk = [], []
        for s_ in range(ns):
            vals = [int(x) for x in rng.integers(1, 1 << 16, size=k * m, dtype=np.uint64)]
            base = s_ * (k + m) * n
            srcs = [buf[base + t * n:base + (t + 1) * n] for t in range(k)]
            rows = buf[base + k * n:base + (k + m) * n]
            jobs.append(fb.Job(ops.Plan.matrix(field, k, m, vals), srcs, rows, n, m, True))
            chk.append((srcs, rows, vals))
        bt = fb.Batch(graphs=True)
        prep = bt.prepare(jobs)
        fn = lambda: bt.run_prepared(prep, stream)
        fn()
        torch.cuda.synchronize()
        ok = all(oracle_matrix_windows(field.ID, chk[i][0], None, [chk[i][1][j * n:(j + 1) * n] for j in range(m)],
                                       chk[i][2], True, rng) for i in (0, ns // 2, ns - 1))
        alg, src_b = ns * (k + m) * n, ns * k * n
        kernel = "batch (Gf16 half-products)" if os.environ.get("FGFC_GF16_HALF", "1") != "0" else "batch (Gf16 tables)"
    elif spec == "uneven":
        res = uneven_batch(dev, max(16, int(args.case_mib)), max(1, args.steps))
        print(json.dumps({"case": args.case, **res}))
        return 0
    else:
        f = fields.Gf8D
        c = [int(x) for x in rng.integers(1, 256, size=4)]
        src = torch.randint(0, 256, (n,), dtype=torch.uint8, device=dev, generator=g)
        dst = torch.randint(0, 256, (4 * n,), dtype=torch.uint8, device=dev, generator=g)
        d0 = dst.clone()
        a, b = 4096, 8192
        if spec == "mul_add":
            fn = lambda: ops.mul_add(f, dst[:n], c[0], src, stream)
            alg, src_b = 3 * n, n
        elif spec == "mul_add_scatter":
            fn = lambda: ops.mul_add_scatter(f, dst, n, c, src, stream)
            alg, src_b = 9 * n, n
        elif spec == "mul_add_gather":
            fn = lambda: ops.mul_add_gather(f, src, c, [dst[j * n:(j + 1) * n] for j in range(4)], stream)
            alg, src_b = 6 * n, 4 * n
        elif spec == "add_assign":
            fn = lambda: ops.add_assign(f, dst[:n], src, stream)
            alg, src_b = 3 * n, n
        else:
            fn = lambda: ops.mul_elementwise(f, dst[:n], src, dst[n:2 * n], stream)
            alg, src_b = 3 * n, 2 * n
        s0 = src.clone()
        fn()
        torch.cuda.synchronize()
        hs, hd = s0[a:b].cpu().numpy().copy(), d0.cpu().numpy()
        if spec == "mul_add":
            w = hd[a:b].copy()
            orc.mul_add(f.ID, w, c[0], hs)
            ok = np.array_equal(dst[a:b].cpu().numpy(), w)
        elif spec == "add_assign":
            ok = np.array_equal(dst[a:b].cpu().numpy(), hd[a:b] ^ hs)
        elif spec == "mul_elementwise":
            w = np.zeros(b - a, np.uint8)
            orc.mul_elementwise(f.ID, w, hs, hd[n + a:n + b].copy())
            ok = np.array_equal(dst[a:b].cpu().numpy(), w)
        kernel = spec
    ms = event_ms(fn, max(1, args.steps), stream, warm=max(0, args.warmup))
    print(json.dumps({"case": args.case, "kernel": kernel, "bytes": n, "ms": round(ms, 4),
                      "GB/s": round(alg / ms / 1e6, 1), "source_GB/s": round(src_b / ms / 1e6, 1),
                      "hbm_frac": round(alg / ms / 1e6 / hbm_peak()[0], 4), "oracle": "passed" if ok else "FAILED"}))
    return 0 if ok else 1


def main():
    args = parse()
    if args.case:
        return run_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    raise SystemExit(main())
