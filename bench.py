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
HASH_NAMES = {"poseidon": 0, "keccak": 1, "poseidonbn128": 2, "poseidon2": 3, "monolith": 4}
# INT32 multiply-class ops per permutation (a 64x64 mulmod counts 10, a
# small-constant MAC 4): Poseidon 1077 mulmod + 1152 MAC, Poseidon2 736 mulmod.
# These two are bound by multiplies, so their op rate is set against the
# measured IMAD issue rate.  Keccak (64-bit logic on the ALU pipe, where one
# LOP3 does a three-input XOR) and Monolith (byte-wise Bars on the ALU pipe,
# concrete layers on the FP64 pipe) are not: an op count set against the IMAD
# rate reads above 1 for them, so the sweep names their bound instead.
OPS_PER_PERM = {0: 15378, 3: 7360}
OTHER_BOUND = {1: "ALU pipe (logic of keccak-f on 32-bit halves; 99 % in ncu)",
               4: "issue (ALU Bars + FP64 concrete layers; 78 % issue in ncu)",
               2: "IMAD pipe (254-bit Montgomery products)"}

# Figures that come from an ncu capture (DRAM bytes per launch, thread
# instructions per permutation) live in profiles/ncu_figures.json together with
# the SHA-256 of the kernel sources they were captured from.  They are reported
# only while the sources still hash to that value; after a kernel change they
# read null until the capture is redone.
PROFILE_FIGURES = ROOT / "profiles" / "ncu_figures.json"


# Host-only orchestration of the batched and served forms: the commit path whose
# kernels the figures describe (zk_lde_leaves_async / zk_lde_async,
# zk_transpose_rev_async, zk_merkle_async) does not run it.
NOT_ON_THE_PROFILED_PATH = {"serve.cu", "admission.h"}


def kernel_sources_sha256() -> str:
    """SHA-256 over the sources that the profiled path's kernels and their launches are built from:
    every zeknox_b200/csrc/*.cu, *.cuh and *.h but NOT_ON_THE_PROFILED_PATH."""
    import hashlib

    h = hashlib.sha256()
    for f in sorted((ROOT / "zeknox_b200" / "csrc").glob("*")):
        if f.suffix in (".cu", ".cuh", ".h") and f.name not in NOT_ON_THE_PROFILED_PATH:
            h.update(f.name.encode())
            h.update(f.read_bytes())
    return h.hexdigest()


def profile_figures() -> dict:
    """{"source": ..., "kernels": {...}} from the capture of the current kernel sources, or {}."""
    if not PROFILE_FIGURES.exists():
        return {}
    d = json.loads(PROFILE_FIGURES.read_text())
    if d.get("sources_sha256") != kernel_sources_sha256():
        return {}
    return d


FIGURES_COMMAND = ('ncu --metrics gpu__time_duration.sum,dram__bytes_read.sum,dram__bytes_write.sum,'
                   'smsp__inst_executed.sum --clock-control none -k regex:"merkle_|ntt_|transpose" -c 60 --csv '
                   '--log-file figures.csv python bench.py --steps 2 --warmup 3 --no-cpu-baseline --sections none')


def write_profile_figures(csv_path, out=None) -> dict:
    """profiles/ncu_figures.json from the CSV launch list of FIGURES_COMMAND:
    the launches of one fused step (the first LDE pass up to the next LDE pass
    after the Merkle kernels) and the plain path's transpose, per launch, stamped
    with the hash of the current kernel sources."""
    import collections
    import csv

    per = collections.OrderedDict()
    hdr = None
    with open(csv_path) as f:
        for r in csv.reader(f):
            if len(r) > 5 and r[0] == "ID":
                hdr = r
                continue
            if hdr and len(r) == len(hdr):
                d = dict(zip(hdr, r))
                e = per.setdefault(int(d["ID"]), {"name": d["Kernel Name"]})
                e[d["Metric Name"]] = float(d["Metric Value"].replace(",", ""))
    launches = list(per.values())
    i = next(i for i, k in enumerate(launches) if "ntt_" in k["name"])
    step = []
    while i < len(launches):
        step.append(launches[i])
        i += 1
        if i < len(launches) and "ntt_" in launches[i]["name"] and any("merkle" in k["name"] for k in step):
            break
    lde = [k for k in step if "ntt_" in k["name"]]
    mk = [k for k in step if "merkle" in k["name"]]
    tr = [k for k in launches if "transpose" in k["name"]]
    b, n_pts = 135, 1 << 18
    perms = n_pts * 17 + 16 * ((n_pts >> 4) - 2) + 16  # leaf sponges of 135 words, inner nodes, cap 4
    dram = lambda ks: sum(k["dram__bytes_read.sum"] + k["dram__bytes_write.sum"] for k in ks)  # noqa: E731
    inst = lambda ks: sum(k["smsp__inst_executed.sum"] for k in ks)  # noqa: E731
    names = lambda ks: [k["name"].split("(")[0][-60:] for k in ks]  # noqa: E731
    fig = {"sources_sha256": kernel_sources_sha256(),
           "sources_note": "hash over zeknox_b200/csrc/*.cu, *.cuh, *.h except " + ", ".join(sorted(NOT_ON_THE_PROFILED_PATH)),
           "command": FIGURES_COMMAND + "; then python bench.py --figures-from figures.csv",
           "kernels": {
               f"merkle poseidon {n_pts}x{b} cap 4": {
                   "dram_bytes_per_launch": dram(mk), "thread_inst_per_perm": inst(mk) * 32 / perms,
                   "launches": names(mk)},
               f"lde_leaves {b}x2^15 rate 3": {
                   "dram_bytes_per_launch": dram(lde), "thread_inst_per_elem": inst(lde) * 32 / (b * n_pts),
                   "launches": names(lde)}}}
    if tr:
        fig["kernels"][f"transpose_rev {b}x2^18"] = {"dram_bytes_per_launch": dram(tr[:1]), "launches": names(tr[:1])}
    Path(out or PROFILE_FIGURES).write_text(json.dumps(fig, indent=1) + "\n")
    return fig


def job_seed(config: int, j: int) -> int:
    """Seed of job j of a multi-job configuration: (0x5EED0000 + config) xor SplitMix64's output for j."""
    z = ((j + 1) * 0x9E3779B97F4A7C15) & (2**64 - 1)
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
    z ^= z >> 31
    return (0x5EED0000 + config) ^ z


def max_over_ranks(values, dist, device) -> list:
    """Each timing is the maximum over the ranks (one all-reduce; identity
    for a single process).  `device` holds the reduction tensor: the rank's
    GPU under NCCL, the CPU under gloo."""
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def replica_throughput(world: int, units_per_step: int, steps: int, ms_max: float) -> float:
    """Whole-job units per second of `world` independent replicas, each doing
    `units_per_step` per step, timed by the slowest rank."""
    return world * units_per_step * steps / (ms_max * 1e-3)


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
    """nvidia-smi clocks / throttle reasons, sampled during the timed region.

    nvidia-smi samples every 20 ms from a moment before the region starts (its
    start-up and NVML initialisation take up to a few hundred ms), and only the
    samples whose timestamps fall inside the region are summarised."""

    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    LEAD_S = 0.4  # sampler running before the region starts

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = ""
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(self.LEAD_S)
        except OSError:
            self.proc = None
        self.t0 = time.time()
        return self

    def __exit__(self, *exc):
        self.t1 = time.time()
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    @staticmethod
    def _stamp(text: str) -> float | None:
        import datetime

        try:
            return datetime.datetime.strptime(text, "%Y/%m/%d %H:%M:%S.%f").timestamp()
        except ValueError:
            return None

    def summary(self) -> dict:
        rows = []
        for ln in (self.out or "").splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((self._stamp(f[0]), float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        inside = [r for r in rows if r[0] is not None and self.t0 is not None and self.t0 <= r[0] <= self.t1]
        use = inside or rows  # no usable timestamps: every sample, flagged below
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = {n for r in use for n, v in zip(names, r[3]) if v.lower() == "active"}
        sm = [r[1] for r in use]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": use[-1][2] if use else None,
                "reasons": sorted(reasons), "samples": len(sm), "interval_ms": 20,
                "window": "timed region" if inside else "whole sampler run"}


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
    ap.add_argument("--workload", default="commit",
                    choices=["commit", "merkle", "sweep", "batched", "served", "fri", "field-ops", "tensor-bound"],
                    help="commit (default, the bench line); the others print their own JSON summary")
    ap.add_argument("--leaves", type=int, default=8192, help="leaf count of the merkle workload (a power of two)")
    ap.add_argument("--streams", type=int, default=4, help="internal streams of a batch / slots of the server")
    ap.add_argument("--budget-gb", type=int, default=120)
    ap.add_argument("--sections", default="batched,served",
                    help="multi-job sections added to the default (commit) line: batched (config 3), served (config 5)")
    ap.add_argument("--batched-jobs", type=int, default=256)
    ap.add_argument("--served-jobs", type=int, default=200, help="prefix of the seeded 10,000-job stream")
    ap.add_argument("--served-rates", type=float, nargs="*", default=[0.75, 1.0],
                    help="arrival rates as fractions of the plain path's measured capacity")
    ap.add_argument("--served-repeats", type=int, default=1)
    ap.add_argument("--served-replay", action="store_true",
                    help="time the plain FIFO arm by a real-time replay at each rate")
    ap.add_argument("--oracle-sample", type=int, default=6, help="jobs per section recomputed on the host")
    ap.add_argument("--figures-from", metavar="CSV",
                    help="write profiles/ncu_figures.json from the launch list of FIGURES_COMMAND, then exit")
    args = ap.parse_args()
    if args.figures_from:
        print(json.dumps(write_profile_figures(args.figures_from)["kernels"]))
        return
    if args.workload != "commit" and args.impl == "ours":
        {"merkle": run_merkle_only, "sweep": run_sweep, "batched": run_batched, "served": run_served,
         "fri": run_fri, "field-ops": run_field_ops, "tensor-bound": run_tensor_bound}[args.workload](args)
        return
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

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
            torch.cuda.synchronize()

    def timed_loop(step, n_phases):
        """W warm-up steps, then K timed steps with an event after each phase."""
        for w in range(args.warmup):
            step(w, None)
        barrier()
        evs = []
        t0e, t1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0e.record(stream)
        for k in range(args.steps):
            e = [torch.cuda.Event(enable_timing=True) for _ in range(n_phases + 1)]
            e[0].record(stream)
            step(k, e)
            evs.append(e)
        t1e.record(stream)
        torch.cuda.synchronize()
        phases = np.array([[e[i].elapsed_time(e[i + 1]) for i in range(n_phases)] for e in evs]).mean(axis=0)
        return t0e.elapsed_time(t1e), [float(x) for x in phases]

    # ---- the timed region: fused commit (LDE written as leaves, then the forest) ----
    def fused_step(i, e):
        zk.lde_leaves(coeffs[i % N_ROT], RATE, out=leaves)
        if e:
            e[1].record(stream)
        zk.merkle_tree(leaves, CAP_H, HASH, digests, cap)
        if e:
            e[2].record(stream)

    launches0 = zk.capi.LIB.zk_kernel_launches()
    with ClockSampler(local) as clk:
        ms, (t_lde, t_mk) = timed_loop(fused_step, 2)
    launches = (zk.capi.LIB.zk_kernel_launches() - launches0) * args.steps // (args.steps + args.warmup)
    cap_dev = cap.cpu().numpy().copy()
    gpu_cap_input = (args.steps - 1) % N_ROT

    # ---- the plain drop-in device path: LDE matrix, transpose, forest ----
    def plain_step(i, e):
        zk.lde(coeffs[i % N_ROT], RATE, out=lde_out)
        if e:
            e[1].record(stream)
        zk.transpose_rev(lde_out, out=leaves)
        if e:
            e[2].record(stream)
        zk.merkle_tree(leaves, CAP_H, HASH, digests, cap)
        if e:
            e[3].record(stream)

    ms_plain, (p_lde, p_tr, p_mk) = timed_loop(plain_step, 3)

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

    # Where an end-to-end step's time goes (untimed pass, host clock per call;
    # each call is synchronous or followed by a synchronize).
    def e2e_phases(i: int):
        t = [time.perf_counter()]
        zk.lde_batch(local, lde_out.data_ptr(), pinned[i % N_ROT].data_ptr(), LG_N, cfg)
        t.append(time.perf_counter())
        zk.transpose_rev_batch(local, leaves.data_ptr(), lde_out.data_ptr(), LG, tcfg)
        t.append(time.perf_counter())
        zk.fill_digests_buf_linear_gpu_with_gpu_ptr(digests.data_ptr(), cap.data_ptr(), leaves.data_ptr(), nd, nc, N,
                                                    B, CAP_H, HASH, local)
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        host_dig.copy_(digests, non_blocking=True)
        host_cap.copy_(cap, non_blocking=True)
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        return np.diff(t) * 1e3

    e2e_ph = np.median(np.array([e2e_phases(k) for k in range(5)]), axis=0)
    e2e_input = (args.steps - 1) % N_ROT

    # ---- max over ranks ----
    ms_max, e2e_max, ms_plain = max_over_ranks([ms, e2e_s, ms_plain], dist, dev)

    if rank == 0:
        value = replica_throughput(world, B * N, args.steps, ms_max)
        e2e_val = world * B * N * args.steps / e2e_max
        peaks = measured_peaks()
        hbm_peak = peaks.get("hbm_gbs")
        int_peak = int32_peak()
        counted = HASH in OPS_PER_PERM  # multiply-bound hashers; the others carry their bound by name
        ops = PERMS * OPS_PER_PERM.get(HASH, 0)
        prof = profile_figures()
        pk = prof.get("kernels", {})
        prof_src = (f"ncu capture of kernel sources sha256 {prof['sources_sha256'][:12]} "
                    f"({prof.get('command', '')})") if prof else None
        sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
        sm_mhz = clk.summary().get("sm_mhz")
        mk_key = f"merkle {HASH_NAME} {N}x{B} cap {CAP_H}"
        lde_key = f"lde_leaves {B}x2^{LG_N} rate {RATE}"
        tr_key = f"transpose_rev {B}x2^{LG}"
        inst = pk.get(mk_key, {}).get("thread_inst_per_perm")
        roof = {
            "kernel": f"Merkle build (leaf sponge + levels + cap), {HASH_NAME}",
            "bound": "int32" if counted else OTHER_BOUND[HASH], "unit": "Gop/s",
            "achieved": ops / (t_mk * 1e-3) / 1e9 if counted else None,
            "peak": int_peak / 1e9 if int_peak else None,
            "frac": (ops / (t_mk * 1e-3)) / int_peak if int_peak and counted else None,
            "traffic": pk.get(mk_key, {}).get("dram_bytes_per_launch"),
            "work_per_launch": (f"{PERMS} {HASH_NAME} permutations x {OPS_PER_PERM[HASH]} INT32 multiply-class ops"
                                if counted else f"{PERMS} {HASH_NAME} permutations"),
            "peak_source": "INT32 IMAD issue rate measured live by zeknox_b200/libzkprobe.so (MEASURED_PEAKS.json "
                           "has no integer figure)",
            "ms_per_launch": t_mk,
            # What the kernel executes, against the SMs' issue rate (4 warp
            # instructions per clock per SM): the op count above assumes the
            # integer form of the MDS layer, which runs on the FP64 pipe here.
            "issue_view": {
                "thread_inst_per_perm": inst,
                "achieved_warp_inst_per_s": inst * PERMS / 32 / (t_mk * 1e-3) if inst else None,
                "peak_warp_inst_per_s": sm_count * 4 * sm_mhz * 1e6 if sm_mhz else None,
                "frac": (inst * PERMS / 32 / (t_mk * 1e-3)) / (sm_count * 4 * sm_mhz * 1e6) if inst and sm_mhz else None,
                "source": prof_src or "no ncu capture of the current kernel sources",
                "peak_source": f"{sm_count} SMs x 4 issue slots x median SM clock sampled in the timed region"},
            # The same kernel against HBM: it reads the leaf matrix once and writes the digests.
            "hbm_view": {"algorithmic_bytes": B * N * 8 + (nd + nc) * 32,
                         "achieved_gbs": (B * N * 8 + (nd + nc) * 32) / (t_mk * 1e-3) / 1e9,
                         "frac": ((B * N * 8 + (nd + nc) * 32) / (t_mk * 1e-3) / 1e9) / hbm_peak if hbm_peak else None,
                         "note": "integer-issue bound, not memory bound: the fraction of HBM is small by nature"},
        }
        hbm_bytes = LDE_BYTES
        roof_hbm = {
            "kernel": "LDE written as leaves (shared-memory NTT passes)", "bound": "hbm", "unit": "GB/s",
            "achieved": hbm_bytes / (t_lde * 1e-3) / 1e9, "peak": hbm_peak,
            "frac": (hbm_bytes / (t_lde * 1e-3) / 1e9) / hbm_peak if hbm_peak else None,
            "traffic": pk.get(lde_key, {}).get("dram_bytes_per_launch"), "algorithmic_bytes": hbm_bytes,
            "ms_per_launch": t_lde,
            "thread_inst_per_output_elem": pk.get(lde_key, {}).get("thread_inst_per_elem"),
            "figures_source": prof_src if lde_key in pk else "no ncu capture of the current kernel sources",
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if hbm_peak else None,
        }
        roof_tr = {
            "kernel": "compute_transpose_rev (bit-reversing column -> leaf transpose, plain path)", "bound": "hbm",
            "unit": "GB/s", "achieved": TRANSPOSE_BYTES / (p_tr * 1e-3) / 1e9, "peak": hbm_peak,
            "frac": (TRANSPOSE_BYTES / (p_tr * 1e-3) / 1e9) / hbm_peak if hbm_peak else None,
            "traffic": pk.get(tr_key, {}).get("dram_bytes_per_launch"), "algorithmic_bytes": TRANSPOSE_BYTES,
            "ms_per_launch": p_tr,
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
                            "fill_digests_buf_linear_gpu_with_gpu_ptr -> D2H digests+cap",
                    "phases_ms": {"lde_with_h2d": float(e2e_ph[0]), "transpose": float(e2e_ph[1]),
                                  "merkle": float(e2e_ph[2]), "d2h": float(e2e_ph[3]),
                                  "note": "median of 5 untimed steps, host clock around each call"}},
            "gpu_launches": int(launches),
            "phases_ms": {"lde_to_leaves": t_lde, "merkle": t_mk},
            "plain_device_path": {"value": world * B * N * args.steps / (ms_plain * 1e-3), "unit": "elems/s",
                                  "ms_per_step": ms_plain / args.steps,
                                  "phases_ms": {"lde": p_lde, "transpose": p_tr, "merkle": p_mk},
                                  "path": "zk_lde_async -> zk_transpose_rev_async -> zk_merkle_async"},
            "roofline": roof,
            "roofline_hbm": roof_hbm,
            "roofline_transpose": roof_tr,
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
        if world == 1:
            # the metric's "batched vs plain" and "p99 latency": configs 3 and 5 in the same line
            secs = [x for x in args.sections.split(",") if x]
            del lde_out, leaves, digests, cap, coeffs
            torch.cuda.empty_cache()
            if "batched" in secs:
                out["batched"] = batched_section(args, zk, torch, not args.no_cpu_baseline)
            if "served" in secs:
                out["served"] = served_section(args, zk, torch, not args.no_cpu_baseline)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# ------------------------------------------------------------------ other workloads
def _field_tensor(zk, torch, elems: int, seed: int):
    """Device tensor of field elements uniform in [0, p): fill_field(seed)."""
    return zk.fill_field(torch.empty(elems, dtype=torch.uint64, device="cuda"), seed)


def _ev_ms(torch, fn, reps=1):
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    for _ in range(reps):
        fn()
    b.record(s)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def run_merkle_only(args):
    """Plain Poseidon Merkle tree, 8192 leaves x 135, cap height 4 (the reference's own CPU-runnable case);
    --leaves picks another power-of-two leaf count of the same width, --hash another hasher."""
    import torch

    import zeknox_b200 as zk

    nl, w, ch = args.leaves, 135, 4
    ht = HASH_NAMES[args.hash]
    assert nl >= 32 and nl & (nl - 1) == 0, "--leaves must be a power of two >= 32"
    host = field_elems(0x5EED0001, nl * w)
    leaves = torch.from_numpy(host).cuda().view(nl, w)
    d, c = zk.merkle_tree(leaves, ch, ht)
    for _ in range(args.warmup):
        zk.merkle_tree(leaves, ch, ht, d, c)
    ms = _ev_ms(torch, lambda: zk.merkle_tree(leaves, ch, ht, d, c), args.steps)
    perms = nl * ((w + (17 if ht == 1 else 8) - 1) // (17 if ht == 1 else 8)) + nl
    out = {"workload": f"merkle {nl}x135 {args.hash} cap_height 4", "ms": ms, "perm_per_s": perms / (ms * 1e-3),
           "leaf_elems_per_s": nl * w / (ms * 1e-3)}
    if args.no_cpu_baseline:
        print(json.dumps(out), flush=True)
        return
    from oracle import oracle as O

    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    t0 = time.perf_counter()
    _, cap_ref = O.ref_merkle_fill(host, w, ch, ht) if O.ref_available() else O.merkle_fill(host, w, ch, ht)
    out["cpu_reference_ms"] = (time.perf_counter() - t0) * 1e3
    out["cap_equals_cpu_reference"] = bool(np.array_equal(cap_ref.reshape(-1, 4), c.cpu().numpy()))
    print(json.dumps(out), flush=True)


def run_sweep(args):
    """Hash sweep: 2^20 leaves x 135, cap height 4, Poseidon / Poseidon2 / Keccak / Monolith / Poseidon-BN128."""
    import torch

    import zeknox_b200 as zk

    nl, w, ch = 1 << 20, 135, 4
    leaves = _field_tensor(zk, torch, nl * w, 0x5EED0004).view(nl, w)
    peak = int32_peak()
    res = {"workload": "merkle sweep 2^20 x 135, cap_height 4", "int32_peak_gops": peak / 1e9 if peak else None}
    for name, ht in (("poseidon", 0), ("poseidon2", 3), ("keccak", 1), ("monolith", 4), ("poseidonbn128", 2)):
        d, c = zk.merkle_tree(leaves, ch, ht)
        for _ in range(args.warmup):
            zk.merkle_tree(leaves, ch, ht, d, c)
        ms = _ev_ms(torch, lambda: zk.merkle_tree(leaves, ch, ht, d, c), max(3, args.steps // 4))
        rate_words = 17 if ht == 1 else 8
        perms = nl * ((w + rate_words - 1) // rate_words) + nl
        ops = perms * OPS_PER_PERM.get(ht, 0)
        res[name] = {"ms": ms, "perm_per_s": perms / (ms * 1e-3), "leaf_elems_per_s": nl * w / (ms * 1e-3),
                     "int32_frac": ops / (ms * 1e-3) / peak if peak and ht in OPS_PER_PERM else None}
        if ht in OTHER_BOUND:
            res[name]["bound"] = OTHER_BOUND[ht]
    if args.no_cpu_baseline:
        print(json.dumps(res), flush=True)
        return
    # zeknox's CPU path on a 2^14-leaf sample of the same shape
    from oracle import oracle as O

    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count()))
    sample = leaves[: 1 << 14].cpu().numpy().reshape(-1)
    for name, ht in (("poseidon", 0), ("poseidon2", 3), ("keccak", 1), ("monolith", 4), ("poseidonbn128", 2)):
        t0 = time.perf_counter()
        (O.ref_merkle_fill if O.ref_available() else O.merkle_fill)(sample, w, ch, ht)
        res[name]["cpu_reference_leaf_elems_per_s"] = (1 << 14) * w / (time.perf_counter() - t0)
    print(json.dumps(res), flush=True)


def run_fri(args):
    """FRI commit phase over a resident GF(p^2) polynomial of 2^15 coefficients at
    rate 3 (2^18 points, the evaluation domain of the default commit), arity 16
    three times, cap height 4, Poseidon; final polynomial of 8 coefficients.
    `ms_with_transcript`: the phase as a prover runs it, a host round trip per
    round for the Fiat-Shamir challenge; `ms_device`: the same kernels with the
    challenges fixed in advance (device time only)."""
    import torch

    import zeknox_b200 as zk

    lg_n, rate, arities, ch = 15, 3, [4, 4, 4], 4
    n = 1 << lg_n
    coeffs = _field_tensor(zk, torch, 2 * n, 0x5EED0006).view(2, n)
    P = zk.P

    def challenge(i, cap):
        return (int(cap.reshape(-1)[0]) % P, int(cap.reshape(-1)[1]) % P)

    for _ in range(args.warmup):
        com = zk.fri_commit(coeffs, rate, arities, ch, challenge)
    betas = [r.beta for r in com.rounds]
    torch.cuda.synchronize()
    reps = max(3, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(reps):
        zk.fri_commit(coeffs, rate, arities, ch, challenge)
    torch.cuda.synchronize()
    ms_t = (time.perf_counter() - t0) * 1e3 / reps

    # Device-only: the same launches with the challenges known in advance.
    bufs = []
    cur_n, shift = n, 7
    for ab in arities:
        N = cur_n << rate
        leaves = torch.empty((N, 2), dtype=torch.uint64, device="cuda")
        nd, nc = zk.merkle_sizes(N >> ab, ch)
        bufs.append((leaves, torch.empty((max(nd, 1), 4), dtype=torch.uint64, device="cuda"),
                     torch.empty((nc, 4), dtype=torch.uint64, device="cuda"),
                     torch.empty((2, cur_n >> ab), dtype=torch.uint64, device="cuda"), shift, ab))
        cur_n >>= ab
        shift = pow(shift, 1 << ab, P)

    def device_phase():
        cur = coeffs
        for (lv, d, c, nxt, sh, ab), beta in zip(bufs, betas):
            zk.lde_leaves_coset(cur, rate, sh, out=lv)
            zk.merkle_tree(lv.view(-1, 2 << ab), ch, 0, d, c)
            zk.fri_fold(cur, ab, beta, out=nxt)
            cur = nxt

    device_phase()
    final_dev = bufs[-1][3].clone()
    ms_d = _ev_ms(torch, device_phase, reps)
    res = {"workload": "fri commit phase: 2^15 GF(p^2) coefficients, rate 3, arity 16 x 3, cap_height 4, poseidon",
           "ms_with_transcript": ms_t, "ms_device": ms_d, "points_per_s": (n << rate) / (ms_d * 1e-3),
           "final_poly_equal": bool(torch.equal(final_dev, com.final_poly))}
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        host = coeffs.cpu().numpy()
        t0 = time.perf_counter()
        _, fin = O.fri_commit(host, rate, arities, ch, challenge)
        res["cpu_port_ms"] = (time.perf_counter() - t0) * 1e3
        res["cpu_port_final_equal"] = bool(np.array_equal(fin, com.final_poly.cpu().numpy()))
    print(json.dumps(res), flush=True)


def _jobs(seed, count, lg_lo, lg_hi, b_lo, b_hi, rates):
    """The seeded job list of a multi-job configuration: (lg_n, polynomials, rate_bits) per job."""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(lg_lo, lg_hi + 1)), int(rng.integers(b_lo, b_hi + 1)), int(rng.choice(rates)))
            for _ in range(count)]


def fifo_latencies(arrivals, service):
    """One server, first in first out: job j starts at max(its arrival, the end of
    job j - 1) and takes service[j].  -> (latency of each job, first arrival to last end)."""
    end, lat = 0.0, []
    for a, sv in zip(arrivals, service):
        end = max(a, end) + sv
        lat.append(end - a)
    return lat, (end - arrivals[0]) if len(lat) else 0.0


def _pct(x, q):
    return float(np.percentile(np.asarray(x, dtype=np.float64), q)) if len(x) else None


class DropIn:
    """One job at a time through a library's zeknox C ABI (this library's, or
    zeknox's own build): compute_batched_lde -> compute_transpose_rev ->
    fill_digests_buf_linear_gpu_with_gpu_ptr on device buffers, then the cap.

    A job whose LDE matrix does not fit the LDE buffer (its footprint, LDE
    matrix plus leaves, exceeds HBM) streams: the LDE and transpose run on
    slices of polynomials, each transposed slice copied into its columns of
    the leaf matrix (cudaMemcpy2DAsync), then the tree of the whole matrix."""

    def __init__(self, torch, lib, check, max_in, max_leaves, max_n, lde_cap, cap_height=4):
        self.torch, self.lib, self.check = torch, lib, check
        self.lde = torch.empty(min(max_leaves, lde_cap), dtype=torch.uint64, device="cuda")
        self.leaves = torch.empty(max_leaves, dtype=torch.uint64, device="cuda")
        self.digests = torch.empty(8 * max_n, dtype=torch.uint64, device="cuda")
        self.cap = torch.empty(4 << cap_height, dtype=torch.uint64, device="cuda")
        self.streamed = 0

    def run(self, coeffs_ptr, lg_n, rate, b, ch, ht=0):
        from zeknox_b200.capi import NTTConfig, TransposeConfig

        torch, L = self.torch, self.lib
        lg = lg_n + rate
        N, n = 1 << lg, 1 << lg_n
        cfg = NTTConfig.default()
        cfg.extension_rate_bits, cfg.with_coset = rate, True
        cfg.are_inputs_on_device = cfg.are_outputs_on_device = True
        t = TransposeConfig.default()
        t.are_inputs_on_device = t.are_outputs_on_device = True
        if b * N <= self.lde.numel():
            cfg.batches, t.batches = b, b
            self.check(L.compute_batched_lde(0, self.lde.data_ptr(), coeffs_ptr, lg_n, 0, cfg))
            self.check(L.compute_transpose_rev(0, self.leaves.data_ptr(), self.lde.data_ptr(), lg, t))
        else:
            self.streamed += 1
            g = self.lde.numel() // (2 * N)  # slice LDE and its transpose side by side in the LDE buffer
            lde, tr = self.lde.data_ptr(), self.lde.data_ptr() + g * N * 8
            for b0 in range(0, b, g):
                nb = min(g, b - b0)
                cfg.batches, t.batches = nb, nb
                self.check(L.compute_batched_lde(0, lde, coeffs_ptr + b0 * n * 8, lg_n, 0, cfg))
                self.check(L.compute_transpose_rev(0, tr, lde, lg, t))
                # rows of nb words -> columns b0 .. b0 + nb of the b-word leaf rows (a strided device copy)
                src = self.lde[g * N: g * N + nb * N].view(N, nb)
                self.leaves[: b * N].view(N, b)[:, b0: b0 + nb].copy_(src)
                torch.cuda.synchronize()
        L.fill_digests_buf_linear_gpu_with_gpu_ptr(self.digests.data_ptr(), self.cap.data_ptr(),
                                                   self.leaves.data_ptr(), 2 * (N - (1 << ch)), 1 << ch, N, b, ch,
                                                   ht, 0)
        cap = self.cap[: 4 << ch].cpu().numpy().copy()  # synchronises the legacy stream the tree ran on
        return cap


def _check_rust(r):
    if r.code != 0:
        raise RuntimeError(f"reference build: code {r.code}")


def ref_gpu_build():
    """zeknox's own sm_100a build (oracle/_ref/libzkref_gpu.so, compiled from its
    sources) through its C ABI, for the baseline leg of the batched workload; None
    when it was not built."""
    import ctypes

    so = ROOT / "oracle" / "_ref" / "libzkref_gpu.so"
    if not so.exists():
        return None
    from zeknox_b200.capi import NTTConfig, RustError, TransposeConfig

    L = ctypes.CDLL(str(so))
    vp, sz, u32, u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64
    for name, args in (("init_twiddle_factors", [sz, sz]), ("init_coset", [sz, sz, u64]),
                       ("compute_batched_lde", [sz, vp, vp, u32, ctypes.c_int, NTTConfig]),
                       ("compute_transpose_rev", [sz, vp, vp, u32, TransposeConfig])):
        getattr(L, name).argtypes = args
        getattr(L, name).restype = RustError
    L.fill_digests_buf_linear_gpu_with_gpu_ptr.argtypes = [vp, vp, vp, u64, u64, u64, u64, u64, u64, u64]
    L.fill_digests_buf_linear_gpu_with_gpu_ptr.restype = None
    return L


def _oracle_caps(sample, cap_height=4):
    """Caps of (seed, lg_n, polys, rate) jobs computed on the host: the oracle's LDE and
    transpose, zeknox's CPU Merkle path when built (else the oracle's)."""
    from oracle import oracle as O

    caps = []
    for seed, lg_n, b, r in sample:
        x = O.fill_field(seed, b << lg_n)
        leaves = O.transpose_rev(O.batch_lde(x, lg_n, r, b), lg_n + r, b)
        fill = O.ref_merkle_fill if O.ref_available() else O.merkle_fill
        caps.append(fill(leaves, b, cap_height, 0)[1].reshape(-1, 4))
    return caps


def batched_section(args, zk, torch, baseline_legs: bool) -> dict:
    """Config 3: 256 jobs, lg_n 12..20, polys 4..200, rate 1..3, cap height 4, Poseidon; inputs
    fill_field(job_seed(3, j)), uniform in [0, p), resident on the device.  Arms, each over every job:
    the plain per-job drop-in path of this library; zk_commit_batch per memory wave (autotuned); the
    same waves as CUDA graphs; and (baseline leg) zeknox's own sm_100a build's per-job drop-in path."""
    jobs = _jobs(0x5EED0003, args.batched_jobs, 12, 20, 4, 200, [1, 2, 3])
    ch = 4
    seeds = [job_seed(3, j) for j in range(len(jobs))]
    offs = np.cumsum([0] + [b << lg for lg, b, _ in jobs])
    inp = torch.empty(int(offs[-1]), dtype=torch.uint64, device="cuda")
    views = []
    for j, (lg, b, r) in enumerate(jobs):
        v = inp[int(offs[j]): int(offs[j + 1])]
        zk.fill_field(v, seeds[j])
        views.append(v.view(b, 1 << lg))
    elems = sum(b << (lg + r) for lg, b, r in jobs)
    mx = max(b << (lg + r) for lg, b, r in jobs)
    mx_n = max(1 << (lg + r) for lg, b, r in jobs)
    max_lg = max(lg + r for lg, _, r in jobs)
    res = {"workload": f"batched commit: {len(jobs)} jobs lg_n 12..20, polys 4..200, rate 1..3, cap_height 4, "
                       "poseidon; inputs fill_field(job seed) resident on the device",
           "jobs": len(jobs), "elems": elems}
    # tables of every size first, for every arm (zeknox's are built by a serial kernel)
    zk.init_coset(0, max_lg, 7)
    for lg in sorted({lg + r for lg, _, r in jobs}):
        zk.init_twiddle_factors(0, lg)
    torch.cuda.synchronize()

    # ---- plain per-job drop-in path of this library
    plain = DropIn(torch, zk.capi.LIB, zk.capi.check, 0, mx, mx_n, mx)
    for (lg, b, r), v in list(zip(jobs, views))[:4]:  # warm-up
        plain.run(v.data_ptr(), lg, r, b, ch)
    torch.cuda.synchronize()
    caps_plain = []
    t0 = time.perf_counter()
    for (lg, b, r), v in zip(jobs, views):
        caps_plain.append(plain.run(v.data_ptr(), lg, r, b, ch))
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    del plain
    torch.cuda.empty_cache()

    # ---- batched: waves of jobs whose outputs fit the budget, one zk_commit_batch each
    budget = args.budget_gb << 30
    order = sorted(range(len(jobs)), key=lambda j: -(jobs[j][1] << (jobs[j][0] + jobs[j][2])))
    waves, cur, used = [], [], 0
    for j in order:
        lg, b, r = jobs[j]
        need = (b << (lg + r)) * 8 + (2 << (lg + r)) * 32
        if cur and used + need > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(j)
        used += need
    waves.append(cur)
    t0 = time.perf_counter()
    tuned = sum(zk.autotune(lg, r, b) > 0 for lg, b, r in jobs)  # outside the timed region
    t_tune = time.perf_counter() - t0
    caps_batch, caps_graph = [None] * len(jobs), [None] * len(jobs)
    t_batch = t_graph = 0.0
    for wave in waves:
        items = [(views[j], jobs[j][2], ch, 0, zk.CommitBuffers(1 << (jobs[j][0] + jobs[j][2]), jobs[j][1], ch))
                 for j in wave]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        zk.commit_batch(items, n_streams=args.streams)
        torch.cuda.synchronize()
        t_batch += time.perf_counter() - t0
        for j, it in zip(wave, items):
            caps_batch[j] = it[4].cap.cpu().numpy()
            it[4].cap.zero_()
        # the same wave captured once into a CUDA graph (capture and the first replay, which maps the
        # graph's memory, outside the timed region), replayed
        g = zk.CommitGraph(items, n_streams=args.streams)
        g.replay()
        for it in items:
            it[4].cap.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.replay()
        torch.cuda.synchronize()
        t_graph += time.perf_counter() - t0
        for j, it in zip(wave, items):
            caps_graph[j] = it[4].cap.cpu().numpy()
        del g, items
        torch.cuda.empty_cache()
    same = lambda a, b: all(np.array_equal(x.reshape(-1), y.reshape(-1)) for x, y in zip(a, b))  # noqa: E731
    res.update({
        "plain": {"elems_per_s": elems / t_plain, "s": t_plain,
                  "path": "per job: compute_batched_lde -> compute_transpose_rev -> "
                          "fill_digests_buf_linear_gpu_with_gpu_ptr -> cap D2H (this library, device buffers)"},
        "batched": {"elems_per_s": elems / t_batch, "s": t_batch, "over_plain": t_plain / t_batch,
                    "waves": len(waves), "streams": args.streams, "budget_gb": args.budget_gb,
                    "autotuned_shape_classes": tuned, "autotune_s": t_tune},
        "graph": {"elems_per_s": elems / t_graph, "s": t_graph, "over_plain": t_plain / t_graph},
        "check": {"batched_caps_equal_plain": same(caps_batch, caps_plain),
                  "graph_caps_equal_plain": same(caps_graph, caps_plain)},
    })
    if baseline_legs:
        # zeknox's own sm_100a build, the same per-job drop-in calls on the same device inputs
        ref = ref_gpu_build()
        if ref is not None:
            for lg in sorted({lg + r for lg, _, r in jobs}):
                _check_rust(ref.init_twiddle_factors(0, lg))
            _check_rust(ref.init_coset(0, max_lg, 7))
            rp = DropIn(torch, ref, _check_rust, 0, mx, mx_n, mx)
            for (lg, b, r), v in list(zip(jobs, views))[:4]:
                rp.run(v.data_ptr(), lg, r, b, ch)
            torch.cuda.synchronize()
            caps_ref = []
            t0 = time.perf_counter()
            for (lg, b, r), v in zip(jobs, views):
                caps_ref.append(rp.run(v.data_ptr(), lg, r, b, ch))
            torch.cuda.synchronize()
            t_ref = time.perf_counter() - t0
            del rp
            torch.cuda.empty_cache()
            res["reference_gpu_plain"] = {
                "elems_per_s": elems / t_ref, "s": t_ref,
                "batched_over_it": t_ref / t_batch, "graph_over_it": t_ref / t_graph, "plain_over_it": t_ref / t_plain,
                "build": "zeknox's CUDA sources compiled for sm_100a (oracle/_ref/libzkref_gpu.so), its per-job "
                         "drop-in path on the same device inputs"}
            res["check"]["plain_caps_equal_reference_gpu"] = same(caps_plain, caps_ref)
        # a sample of the smallest jobs recomputed on the host
        small = sorted(range(len(jobs)), key=lambda j: jobs[j][1] << (jobs[j][0] + jobs[j][2]))[: args.oracle_sample]
        want = _oracle_caps([(seeds[j], jobs[j][0], jobs[j][1], jobs[j][2]) for j in small])
        res["check"]["sample_caps_equal_oracle"] = same([caps_plain[j] for j in small], want)
        res["check"]["oracle_sample"] = f"{len(small)} smallest jobs: host LDE + transpose by the oracle, Merkle " \
                                        f"by zeknox's CPU path"
    del inp, views
    torch.cuda.empty_cache()
    return res


def served_section(args, zk, torch, baseline_legs: bool) -> dict:
    """Config 5: the first `served_jobs` jobs of the seeded 10,000-job stream (lg_n 12..22, polys 8..300,
    rate 3, cap height 4, Poseidon; inputs fill_field(job_seed(5, j)), generated on the device as each job
    starts), Poisson arrivals at fractions of the plain path's capacity.

    plain: the drop-in per-job path, one job at a time in arrival order (FIFO).  Each job's service time is
    measured once, back to back in arrival order; the FIFO latencies at each rate follow from those times
    and the arrival times (start = max(arrival, previous end)), or, with --served-replay, from a real-time
    replay of the queue.  served: zk_server (120 GB budget, 4 slots), real time, seeded submissions.
    --served-repeats R repeats both arms (service pass and served runs) on the same arrival schedule and
    reports the medians and every run."""
    n_jobs = args.served_jobs
    ch, r = 4, 3
    jobs = _jobs(0x5EED0005, 10000, 12, 22, 8, 300, [3])[:n_jobs]
    seeds = [job_seed(5, j) for j in range(n_jobs)]
    elems = sum(b << (lg + r) for lg, b, _ in jobs)
    mx_in = max(b << lg for lg, b, _ in jobs)
    mx = max(b << (lg + r) for lg, b, _ in jobs)
    mx_n = max(1 << (lg + r) for lg, _, _ in jobs)
    zk.init_coset(0, max(lg for lg, _, _ in jobs) + r, 7)
    for lg in sorted({lg + r for lg, _, _ in jobs}):
        zk.init_twiddle_factors(0, lg)
    # the LDE -> leaves plan of every shape class of the stream, tuned before either arm runs (the
    # plain arm's row LDE has no tuned choices); outside every timed region
    t0 = time.perf_counter()
    tuned = sum(zk.autotune(lg, r, b) > 0 for lg, b, _ in jobs)
    t_tune = time.perf_counter() - t0

    def service_pass():
        """Every job through the drop-in path, back to back in arrival order: per-job service times (input
        generation included, as in a served job) and caps."""
        dev_in = torch.empty(mx_in, dtype=torch.uint64, device="cuda")
        # the LDE matrix of a job up to 60 GB; larger ones stream (leaves up to 80.5 GB beside it)
        plain = DropIn(torch, zk.capi.LIB, zk.capi.check, mx_in, mx, mx_n, (60 << 30) // 8)

        def plain_job(j):
            lg, b, _ = jobs[j]
            zk.fill_field(dev_in[: b << lg], seeds[j])
            return plain.run(dev_in.data_ptr(), lg, r, b, ch)

        plain_job(0)
        torch.cuda.synchronize()
        service, caps = [], []
        with ClockSampler(torch.cuda.current_device()) as clk:
            for j in range(n_jobs):
                t0 = time.perf_counter()
                caps.append(plain_job(j))
                service.append(time.perf_counter() - t0)
        return service, caps, clk.summary(), plain.streamed, plain_job, (plain, dev_in)

    def served_run(arr):
        with zk.Server(hbm_budget_bytes=args.budget_gb << 30, slots=args.streams) as srv:
            lat_s, caps_s, errs, tick, split = {}, {}, [], {}, {}

            def client():  # completions in order; each tree released at once
                try:
                    while len(lat_s) < n_jobs:
                        t = srv.wait_any(timeout_ms=1000)
                        if t is not None:
                            cap, lat = srv.wait(t)
                            lat_s[t], caps_s[t] = lat, cap
                            split[t] = srv.job_times(t)
                            srv.release(t)
                except Exception as e:  # noqa: BLE001 - reported by the main thread
                    errs.append(e)

            th = threading.Thread(target=client)
            with ClockSampler(torch.cuda.current_device()) as clk:
                th.start()
                t0 = time.perf_counter()
                for j, a in enumerate(arr):
                    now = time.perf_counter() - t0
                    if now < a:
                        time.sleep(a - now)
                    lg, b, _ = jobs[j]
                    tick[j] = srv.submit_seeded(seeds[j], lg, b, r, ch)
                th.join()
            if errs:
                raise errs[0]
            span = time.perf_counter() - t0 - arr[0]
            st = srv.stats()
        lats = [lat_s[tick[j]] for j in range(n_jobs)]
        caps = [caps_s[tick[j]] for j in range(n_jobs)]
        slow = sorted(range(n_jobs), key=lambda j: -lats[j])[: max(1, n_jobs // 100)]
        return {"p50_s": _pct(lats, 50), "p99_s": _pct(lats, 99), "elems_per_s": elems / span,
                "started_ahead": st["ahead"], "max_queue": st["max_queue"],
                "hbm_peak_gb": st["hbm_peak"] / 2**30, "alloc_max_s": st["alloc_max_s"],
                "pool_gb": [st["pool_reserved_start"] / 2**30, st["pool_reserved_high"] / 2**30],
                # the slowest 1 %: job, lg_n, polys, latency, seconds queued, seconds running
                "slowest": [[j, jobs[j][0], jobs[j][1], round(lats[j], 4), *(round(x, 4) for x in split[tick[j]])]
                            for j in slow],
                "clocks": clk.summary()}, caps

    arrivals, res, caps_ref = None, None, None
    runs = {f: {"plain": [], "served": []} for f in args.served_rates}
    all_caps_ok = True
    for rep in range(args.served_repeats):
        service, caps_plain, clk_plain, streamed, plain_job, bufs = service_pass()
        if arrivals is None:  # one arrival schedule for every repeat, from the first capacity measurement
            cap_jobs_per_s = n_jobs / sum(service)
            rng = np.random.default_rng(0x5EED0055)
            arrivals = {f: np.cumsum(rng.exponential(1.0 / (f * cap_jobs_per_s), n_jobs))
                        for f in args.served_rates}
            caps_ref = caps_plain
            res = {"workload": f"served: first {n_jobs} jobs of the seeded 10,000-job stream (lg_n 12..22, polys "
                               "8..300, rate 3, cap_height 4, poseidon); inputs fill_field(job seed) generated on "
                               "the device at each job's start (both arms)",
                   "jobs": n_jobs, "elems": elems, "plain_capacity_jobs_per_s": cap_jobs_per_s,
                   "plain_capacity_elems_per_s": elems / sum(service), "plain_streamed_jobs": streamed,
                   "plain_service_s": {"p50": _pct(service, 50), "p99": _pct(service, 99), "max": max(service)},
                   "plain_service_clocks": clk_plain,
                   "slots": args.streams, "budget_gb": args.budget_gb, "autotuned_shape_classes": tuned,
                   "autotune_s": t_tune, "repeats": args.served_repeats, "rates": {}}
        all_caps_ok &= all(np.array_equal(x.reshape(-1), y.reshape(-1)) for x, y in zip(caps_plain, caps_ref))
        for f in args.served_rates:
            if args.served_replay:  # the FIFO queue in real time
                lat = []
                t0 = time.perf_counter()
                for j, a in enumerate(arrivals[f]):
                    now = time.perf_counter() - t0
                    if now < a:
                        time.sleep(a - now)
                    plain_job(j)
                    lat.append(time.perf_counter() - t0 - a)
                lat_p, span_p = lat, time.perf_counter() - t0 - arrivals[f][0]
            else:
                lat_p, span_p = fifo_latencies(arrivals[f], service)
            runs[f]["plain"].append({"p50_s": _pct(lat_p, 50), "p99_s": _pct(lat_p, 99), "elems_per_s": elems / span_p})
        del bufs, plain_job
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        for f in args.served_rates:
            one, caps_s = served_run(arrivals[f])
            all_caps_ok &= all(np.array_equal(x.reshape(-1), y.reshape(-1)) for x, y in zip(caps_s, caps_ref))
            runs[f]["served"].append(one)
            print(json.dumps({"repeat": rep, "rate": f, "plain": runs[f]["plain"][-1], "served": one}),
                  file=sys.stderr, flush=True)
    med = lambda xs, k: float(np.median([x[k] for x in xs]))  # noqa: E731
    for f in args.served_rates:
        P, S = runs[f]["plain"], runs[f]["served"]
        entry = {
            "arrival_jobs_per_s": f * res["plain_capacity_jobs_per_s"],
            "plain": {"p50_s": med(P, "p50_s"), "p99_s": med(P, "p99_s"), "elems_per_s": med(P, "elems_per_s"),
                      "how": "real-time replay of the FIFO queue" if args.served_replay
                      else "FIFO queue over the measured per-job service times"},
            "served": {"p50_s": med(S, "p50_s"), "p99_s": med(S, "p99_s"), "elems_per_s": med(S, "elems_per_s"),
                       "started_ahead": int(med(S, "started_ahead")), "max_queue": int(med(S, "max_queue")),
                       "hbm_peak_gb": med(S, "hbm_peak_gb"), "clocks": S[len(S) // 2]["clocks"]},
        }
        entry["served_over_plain"] = {"p50": entry["plain"]["p50_s"] / entry["served"]["p50_s"],
                                      "p99": entry["plain"]["p99_s"] / entry["served"]["p99_s"],
                                      "elems_per_s": entry["served"]["elems_per_s"] / entry["plain"]["elems_per_s"]}
        if len(S) > 1:  # run-to-run spread, both arms
            entry["runs"] = {"plain": [{k: x[k] for k in ("p50_s", "p99_s", "elems_per_s")} for x in P],
                             "served": [{k: x[k] for k in ("p50_s", "p99_s", "elems_per_s")} for x in S]}
        res["rates"][str(f)] = entry
    res["check"] = {"served_caps_equal_plain": bool(all_caps_ok)}
    if baseline_legs:
        small = sorted(range(n_jobs), key=lambda j: jobs[j][1] << jobs[j][0])[: args.oracle_sample]
        want = _oracle_caps([(seeds[j], jobs[j][0], jobs[j][1], r) for j in small])
        res["check"]["sample_caps_equal_oracle"] = all(np.array_equal(caps_ref[j].reshape(-1), w.reshape(-1))
                                                       for j, w in zip(small, want))
    return res


def run_field_ops(args):
    """One launch per field operation (libzkprobe.so), for counting instructions per operation under ncu:
    the kernel's count minus probe_base's (probe_dft8: minus probe_dft8_base's), divided by the iterations."""
    import ctypes

    lib = ctypes.CDLL(str(ROOT / "zeknox_b200" / "libzkprobe.so"))
    iters = 4096
    r = lib.zk_probe_field_ops(iters)
    assert r == 0, r
    print(json.dumps({"workload": "field-ops", "iterations": iters}), flush=True)


def run_tensor_bound(args):
    """What an int8 tensor-core formulation would cost in its GEMM alone, measured with the library int8
    GEMM (cuBLASLt through torch._int_mm: int8 x int8 -> int32), at the shapes the default commit needs:

    * LDE: a 64-point DFT over byte limbs.  A line of 64 elements is 64 x 8 bytes (K = 512); the DFT matrix's
      entries are powers of two, so each output element needs 12 partial sums (one per byte position of a
      96-bit result, 2^96 = -1 folding the rest): N = 64 x 12 = 768.  The 135 x 2^18 output is 552,960 lines
      per 64-point level, and the transform has three such levels.
    * Poseidon: the MDS layer of one round over byte limbs of the 12 lanes (K = 96, N = 96) for the
      4,456,448 leaf permutations; a permutation has 30 rounds.

    Both GEMMs write their int32 partial sums to HBM here; a fused kernel would keep them in TMEM, so the
    GEMM time is the compute floor of each formulation, before its recombination arithmetic.  Beside each:
    the SIMT kernel's measured time for the same work in the default commit."""
    import torch

    import zeknox_b200 as zk

    def ev(fn, reps=10):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    out = {"workload": "tensor-core bound: int8 GEMMs of the byte-limb formulations (cuBLASLt via torch._int_mm)"}
    g = torch.Generator(device="cuda").manual_seed(1)
    for name, (m, k, n, reps_per_commit) in {"lde_dft64_level": (552960, 512, 768, 3),
                                             "poseidon_mds_round": (4456448, 96, 96, 30)}.items():
        a = torch.randint(-128, 127, (m, k), generator=g, device="cuda", dtype=torch.int8)
        b = torch.randint(-128, 127, (k, n), generator=g, device="cuda", dtype=torch.int8)
        try:
            torch._int_mm(a, b)
        except RuntimeError:  # some builds want the second operand column-major
            b = b.t().contiguous().t()
        ms = ev(lambda: torch._int_mm(a, b))
        out[name] = {"m": m, "k": k, "n": n, "gemm_ms": ms, "tops": 2 * m * k * n / (ms * 1e-3) / 1e12,
                     "per_commit": reps_per_commit, "gemm_ms_per_commit": ms * reps_per_commit}
        del a, b
        torch.cuda.empty_cache()
    x = zk.fill_field(torch.empty(135 << 15, dtype=torch.uint64, device="cuda"), 7).view(135, 1 << 15)
    lv = torch.empty((1 << 18, 135), dtype=torch.uint64, device="cuda")
    out["simt_lde_to_leaves_ms"] = ev(lambda: zk.lde_leaves(x, 3, out=lv))
    d, c = zk.merkle_tree(lv, 4, 0)
    out["simt_merkle_ms"] = ev(lambda: zk.merkle_tree(lv, 4, 0, d, c))
    print(json.dumps(out), flush=True)


def run_batched(args):
    import torch

    import zeknox_b200 as zk

    print(json.dumps(batched_section(args, zk, torch, not args.no_cpu_baseline)), flush=True)


def run_served(args):
    import torch

    import zeknox_b200 as zk

    print(json.dumps(served_section(args, zk, torch, not args.no_cpu_baseline)), flush=True)


if __name__ == "__main__":
    main()
