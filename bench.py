#!/usr/bin/env python
"""Benchmark of the Goldilocks polynomial commitment on B200.

Workload (one step): 135 polynomials of 2^15 coefficients -> coset LDE with
rate_bits 3 (2^18 evaluations each, coset shift 7) -> bit-reversing transpose
to 2^18 leaves x 135 elements -> Poseidon Merkle tree with cap height 4.
Metric: committed LDE evaluations per second (135 * 2^18 per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs one independent replica per GPU (the commit does not shard across
GPUs: "replicas only"); launch it with torch.distributed.run.  Rank 0 prints
one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Goldilocks LDE+Merkle commit elems/s, batched vs plain, bit-exact; p99 latency"
P = 0xFFFFFFFF00000001
HASH_NAMES = {"poseidon": 0, "keccak": 1, "poseidon2": 3}
# INT32 multiply-class ops per permutation (a 64x64 mulmod counts 10, a
# small-constant MAC 4): Poseidon 1077 mulmod + 1152 MAC, Poseidon2 736 mulmod,
# Keccak-f 3720 64-bit logic ops counted as 2 each.
OPS_PER_PERM = {0: 15378, 3: 7360, 1: 7440}


def set_workload(polys=135, lg_n=15, rate=3, cap_h=4, hash_name="poseidon", rot=4):
    """Workload of one step; the defaults are the plain single-job commit
    (135 x 2^15 coefficients, rate 3, Poseidon, cap height 4)."""
    global B, LG_N, RATE, CAP_H, LG, N, n, HASH, HASH_NAME, N_ROT, WORKLOAD, LEAF_PERMS, NODE_PERMS, PERMS
    global LDE_BYTES, TRANSPOSE_BYTES
    B, LG_N, RATE, CAP_H, HASH_NAME, N_ROT = polys, lg_n, rate, cap_h, hash_name, rot
    HASH = HASH_NAMES[hash_name]
    LG = LG_N + RATE
    N, n = 1 << LG, 1 << LG_N
    WORKLOAD = (f"commit: LDE {B}x2^{LG_N} rate {RATE} coset 7 -> transpose_rev -> {hash_name} Merkle "
                f"cap_height {CAP_H}")
    rate_words = 17 if HASH == 1 else 8  # elements absorbed per permutation
    LEAF_PERMS = N * ((B + rate_words - 1) // rate_words)
    NODE_PERMS = (1 << CAP_H) * ((N >> CAP_H) - 2) + (1 << CAP_H)  # internal nodes + cap entries
    PERMS = LEAF_PERMS + NODE_PERMS
    LDE_BYTES = 8 * B * (n + N)
    TRANSPOSE_BYTES = 16 * B * N


set_workload()


def field_elems(seed: int, count: int) -> np.ndarray:
    """SplitMix64 stream rejection-sampled to [0, p)."""
    out, s = [], seed
    have = 0
    while have < count:
        idx = np.arange(1, count - have + 4097, dtype=np.uint64)
        with np.errstate(over="ignore"):
            z = np.uint64(s) + idx * np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z ^= z >> np.uint64(31)
        z = z[z < np.uint64(P)]
        out.append(z)
        have += z.size
        s = (s * 0x9E3779B97F4A7C15 + 1) & (2**64 - 1)
    return np.ascontiguousarray(np.concatenate(out)[:count])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons, sampled during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in (self.out or "").splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for name, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return json.loads(p.read_text())
    return {}


def int32_peak() -> float | None:
    import ctypes

    so = ROOT / "zeknox_b200" / "libzkprobe.so"
    if not so.exists():
        return None
    lib = ctypes.CDLL(str(so))
    lib.zk_probe_imad_ops_per_s.restype = ctypes.c_double
    lib.zk_probe_imad_ops_per_s.argtypes = [ctypes.c_int]
    v = lib.zk_probe_imad_ops_per_s(5)
    return v if v > 0 else None


# ------------------------------------------------------------------ CPU legs
def cpu_commit(coeffs: np.ndarray):
    """zeknox's CPU path for the same step: the oracle's LDE and transpose
    (zeknox has no CPU LDE) and zeknox's own fill_digests_buf_linear_cpu (when
    built in oracle/_ref) for the Merkle tree.  Returns (cap, kind)."""
    from oracle import oracle as O

    lde = O.batch_lde(coeffs, LG_N, RATE, B)
    leaves = O.transpose_rev(lde, LG, B)
    if O.ref_available():
        _, cap = O.ref_merkle_fill(leaves, B, CAP_H, HASH)
        return cap, "reference"
    _, cap = O.merkle_fill(leaves, B, CAP_H, HASH)
    return cap, "port"


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    coeffs = [field_elems(0x5EED0002 + r, B * n) for r in range(2)]
    for w in range(args.warmup):
        cpu_commit(coeffs[w % 2])
    t0 = time.perf_counter()
    kind = "port"
    for k in range(args.steps):
        _, kind = cpu_commit(coeffs[k % 2])
    dt = time.perf_counter() - t0
    v = B * N * args.steps / dt
    sample = ("full step on the host: LDE+transpose by the oracle port (zeknox has no CPU LDE), Merkle by "
              + ("zeknox's own fill_digests_buf_linear_cpu (oracle/_ref)" if kind == "reference" else "the oracle port"))
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "elems/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64 (GF(p), p = 2^64 - 2^32 + 1)", "data": "synthetic",
        "config": {"workload": WORKLOAD, "polys": B, "lg_n": LG_N, "rate_bits": RATE, "cap_height": CAP_H,
                   "hash": HASH_NAME, "threads": int(os.environ["OMP_NUM_THREADS"])},
        "cpu_baseline": {"value": v, "unit": "elems/s", "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": kind,
                         "sample": sample},
        "e2e": {"value": v, "unit": "elems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


# ------------------------------------------------------------------ GPU arm
def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--polys", type=int, default=135, help="polynomials (leaf width)")
    ap.add_argument("--lg-n", type=int, default=15, help="log2 coefficients per polynomial")
    ap.add_argument("--rate-bits", type=int, default=3)
    ap.add_argument("--cap-height", type=int, default=4)
    ap.add_argument("--hash", default="poseidon", choices=sorted(HASH_NAMES))
    args = ap.parse_args()
    set_workload(args.polys, args.lg_n, args.rate_bits, args.cap_height, args.hash)
    if args.impl == "reference":
        run_reference(args)
        return
    assert args.warmup >= 3, "at least 3 warm-up steps"

    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    import zeknox_b200 as zk

    dev = torch.device("cuda", local)
    host_coeffs = [field_elems(0x5EED0002 + r, B * n) for r in range(N_ROT)]
    coeffs = [torch.from_numpy(c).to(dev).view(B, n) for c in host_coeffs]
    lde_out = torch.empty((B, N), dtype=torch.uint64, device=dev)
    leaves = torch.empty((N, B), dtype=torch.uint64, device=dev)
    nd, nc = zk.merkle_sizes(N, CAP_H)
    digests = torch.empty((nd, 4), dtype=torch.uint64, device=dev)
    cap = torch.empty((nc, 4), dtype=torch.uint64, device=dev)
    stream = torch.cuda.current_stream()

    ev = {}

    def step(i: int, timed: bool = False):
        if timed:
            ev.setdefault("e", []).append([torch.cuda.Event(enable_timing=True) for _ in range(4)])
            e = ev["e"][-1]
            e[0].record(stream)
        zk.lde(coeffs[i % N_ROT], RATE, out=lde_out)
        if timed:
            e[1].record(stream)
        zk.transpose_rev(lde_out, out=leaves)
        if timed:
            e[2].record(stream)
        zk.merkle_tree(leaves, CAP_H, HASH, digests, cap)
        if timed:
            e[3].record(stream)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    for w in range(args.warmup):
        step(w)
    barrier()
    launches0 = zk.capi.LIB.zk_kernel_launches()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        t_start.record(stream)
        for k in range(args.steps):
            step(k, timed=True)
        t_end.record(stream)
        torch.cuda.synchronize()
    launches = zk.capi.LIB.zk_kernel_launches() - launches0
    ms = t_start.elapsed_time(t_end)
    phase = np.array([[e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2]), e[2].elapsed_time(e[3])] for e in ev["e"]])
    t_lde, t_tr, t_mk = (float(x) for x in phase.mean(axis=0))
    cap_dev = cap.cpu().numpy().copy()
    gpu_cap_input = (args.steps - 1) % N_ROT

    # ---- end to end through the C ABI with host buffers ----
    pinned = [torch.from_numpy(c).pin_memory() for c in host_coeffs]
    host_dig = torch.empty((nd, 4), dtype=torch.uint64).pin_memory()
    host_cap = torch.empty((nc, 4), dtype=torch.uint64).pin_memory()
    cfg = zk.NTTConfig.default()
    cfg.batches, cfg.extension_rate_bits, cfg.with_coset = B, RATE, True
    cfg.are_inputs_on_device, cfg.are_outputs_on_device = False, True
    tcfg = zk.TransposeConfig.default()
    tcfg.batches, tcfg.are_inputs_on_device, tcfg.are_outputs_on_device = B, True, True

    def e2e_step(i: int):
        zk.lde_batch(local, lde_out.data_ptr(), pinned[i % N_ROT].data_ptr(), LG_N, cfg)
        zk.transpose_rev_batch(local, leaves.data_ptr(), lde_out.data_ptr(), LG, tcfg)
        zk.fill_digests_buf_linear_gpu_with_gpu_ptr(digests.data_ptr(), cap.data_ptr(), leaves.data_ptr(), nd, nc, N,
                                                    B, CAP_H, HASH, local)
        host_dig.copy_(digests, non_blocking=True)
        host_cap.copy_(cap, non_blocking=True)
        torch.cuda.synchronize()

    for w in range(args.warmup):
        e2e_step(w)
    barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        e2e_step(k)
    barrier()
    e2e_s = time.perf_counter() - t0
    cap_e2e = host_cap.numpy().copy()
    e2e_input = (args.steps - 1) % N_ROT

    # ---- max over ranks ----
    ms_t = torch.tensor([ms, e2e_s], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max, e2e_max = float(ms_t[0]), float(ms_t[1])

    if rank == 0:
        value = world * B * N * args.steps / (ms_max * 1e-3)
        e2e_val = world * B * N * args.steps / e2e_max
        peaks = measured_peaks()
        hbm_peak = peaks.get("hbm_gbs")
        int_peak = int32_peak()
        ops = PERMS * OPS_PER_PERM[HASH]
        roof = {
            "kernel": f"Merkle build (leaf sponge + levels + cap), {HASH_NAME}",
            "bound": "int32", "unit": "Gop/s",
            "achieved": ops / (t_mk * 1e-3) / 1e9,
            "peak": int_peak / 1e9 if int_peak else None,
            "frac": (ops / (t_mk * 1e-3)) / int_peak if int_peak else None,
            "traffic": None,
            "work_per_launch": f"{PERMS} {HASH_NAME} permutations x {OPS_PER_PERM[HASH]} INT32 multiply-class ops",
            "peak_source": "INT32 IMAD issue rate measured live by zeknox_b200/libzkprobe.so (MEASURED_PEAKS.json "
                           "has no integer figure)",
            "ms_per_launch": t_mk,
        }
        hbm_bytes = LDE_BYTES + TRANSPOSE_BYTES
        roof_hbm = {
            "kernel": "LDE (2 shared-memory passes) + transpose_rev", "bound": "hbm", "unit": "GB/s",
            "achieved": hbm_bytes / ((t_lde + t_tr) * 1e-3) / 1e9, "peak": hbm_peak,
            "frac": (hbm_bytes / ((t_lde + t_tr) * 1e-3) / 1e9) / hbm_peak if hbm_peak else None,
            "traffic": None, "algorithmic_bytes": hbm_bytes, "ms_lde": t_lde, "ms_transpose": t_tr,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm_peak else None,
        }
        out = {
            "metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 (GF(p), p = 2^64 - 2^32 + 1)",
            "data": "synthetic (SplitMix64 seeded, uniform in [0,p))",
            "config": {"workload": WORKLOAD, "polys": B, "lg_n": LG_N, "rate_bits": RATE, "cap_height": CAP_H,
                       "hash": HASH_NAME, "parallelism": f"replicas x{world}",
                       "l2": f"inputs rotated over {N_ROT} buffers ({N_ROT * B * n * 8 >> 20} MiB > L2); per-step "
                             f"working set {(B * n + 2 * B * N + 4 * nd) * 8 >> 20} MiB"},
            "e2e": {"value": e2e_val, "unit": "elems/s", "h2d_bytes_per_step": B * n * 8,
                    "d2h_bytes_per_step": (nd + nc) * 32,
                    "path": "compute_batched_lde (pinned host in) -> compute_transpose_rev -> "
                            "fill_digests_buf_linear_gpu_with_gpu_ptr -> D2H digests+cap"},
            "gpu_launches": int(launches),
            "phases_ms": {"lde": t_lde, "transpose": t_tr, "merkle": t_mk},
            "roofline": roof,
            "roofline_hbm": roof_hbm,
            "clocks": clk.summary(),
            "check": {"cap_device_path_equals_c_abi_path": bool(np.array_equal(cap_dev, cap_e2e))
                      if gpu_cap_input == e2e_input else None},
        }
        if world == 1 and not args.no_cpu_baseline:
            os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
            t0 = time.perf_counter()
            cpu_cap, kind = cpu_commit(host_coeffs[e2e_input])
            dt = time.perf_counter() - t0
            out["cpu_baseline"] = {
                "value": B * N / dt, "unit": "elems/s", "cores": int(os.environ["OMP_NUM_THREADS"]), "kind": kind,
                "sample": "one full step on the host: LDE+transpose by the oracle port (zeknox has no CPU LDE); "
                          "Merkle by " + ("zeknox's fill_digests_buf_linear_cpu" if kind == "reference"
                                          else "the oracle port"),
            }
            out["check"]["cap_equals_cpu_reference"] = bool(np.array_equal(cpu_cap.reshape(-1, 4), cap_e2e))
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
