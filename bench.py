#!/usr/bin/env python
"""Benchmark of the plain SIMBA search (candidate-evals/s) on B200.

Workload (one GPU): the larger plain-search configuration -- a target over 3
variables + the constant 1 (4 terminals), 64 uniform uint64 samples
(SplitMix64 seed 1) -- with the outputs replaced by random words so that no
expression matches and every candidate of sizes 2..L is evaluated (L = 14 by
default: 9.7e11 candidates per step).  A step is one sweep of those sizes:
exactly the blocks the reference launches for `simba <instance> L+1`.

value     candidates / second with samples and value tables resident in HBM
          (session API), timed with CUDA events on the launching stream.
e2e       the same metric through simba_solve() from host buffers: H2D of the
          samples, table build, search, D2H of the result, every step.
roofline  the search kernel's integer lane-operations (nested compares: the
          masked compare and explicitly evaluated levels per candidate; hash
          join: hash and filter test per bottom value and context block) over
          the measured int32 issue peak of the device (simba_int_peak).
cpu_baseline  the OpenMP oracle (a port of the reference's per-rank
          unrank + evaluate) on a bounded sample of size-L ranks.

--impl reference runs the reference's own CUDA executable (rebuilt for
sm_100a into oracle/_ref/) on the uint32 version of the same workload,
sweeping sizes 2..13, and reports its candidate-evals/s from its own timer
minus the CUDA context start-up it also times.

Multi-GPU: one process per GPU (torchrun); every rank sweeps its own
independent instance (seed 1 + rank), no data-path collective: weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SWEEP_L = 14
REF_L = 13
N_VARS, N_SAMPLES, TARGET_SIZE = 3, 64, 15


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="simba_b200", choices=["simba_b200", "reference"])
    ap.add_argument("--sweep", type=int, default=SWEEP_L)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--case", choices=["spine12", "batch10", "vfb10"],
                    help="run one small profiling case instead of the benchmark (no JSON line)")
    return ap.parse_args()


def run_case(name: str) -> None:
    """Small cases for ncu captures (see profiles/): a size-12 sweep of the
    benchmark instance run twice; a 256-instance mixed batch to max size 11
    (its 9th spine launch is the size-10 round); VFB to maxLen 10 on the
    benchmark instance."""
    sys.path.insert(0, str(ROOT))
    import simba_b200 as S
    from simba_b200.instances import iter_batch, make_instance
    inst = make_instance(TARGET_SIZE, N_VARS, N_SAMPLES, 1, word_bits=64, unsat=True)
    if name == "spine12":
        with S.Session(inst) as ss:
            for _ in range(2):
                r = ss.sweep(12, 12)
        print("spine12", r.candidates, r.evaluated, r.kernel_ms)
    elif name == "batch10":
        insts = list(iter_batch(256, 5 * 10 ** 6, sizes=range(7, 20), vars_=(2, 3, 4, 5),
                                samples=(32, 64, 128), word_bits=64))
        res, st = S.solve_batch(insts, 11, table_bytes=12 << 20, budget=60)
        print("batch10", st["rounds"], st["evaluated"], st["kernel_ms"], st["solved"])
    else:
        r = S.vfb_solve(inst, 10, budget=120)
        print("vfb10", r.status, r.candidates, r.rows_total, r.device_ms)


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(seed: int, bits: int):
    from simba_b200.instances import make_instance
    return make_instance(TARGET_SIZE, N_VARS, N_SAMPLES, seed, word_bits=bits, const_one=True,
                         unsat=True)


def sweep_candidates(k: int, lo: int, hi: int) -> int:
    from simba_b200 import count_table
    t = count_table(hi, k)
    return int(sum(int(t[s][8]) for s in range(lo, hi + 1)))


def cpu_baseline(inst, size: int) -> dict:
    """OpenMP oracle on a bounded sample of size-`size` ranks (~10-20 s)."""
    from oracle import oracle as O
    cores = O.max_threads()
    probe = 2_000_000
    t0 = time.perf_counter()
    O.scan_range(inst.inputs, inst.outputs, size, 0, probe, 64)
    rate = probe / max(time.perf_counter() - t0, 1e-6)
    n = int(min(max(rate * 12, probe), 2e10))  # about 12 s of CPU work
    t0 = time.perf_counter()
    ev, _, _ = O.scan_range(inst.inputs, inst.outputs, size, 0, n, 64)
    dt = time.perf_counter() - t0
    return {"value": ev / dt, "unit": "candidate-evals/s", "cores": cores, "kind": "port",
            "sample": f"first {ev} ranks of size {size}, {N_SAMPLES} uint64 samples, "
                      f"{N_VARS} vars + const 1, unsatisfiable target ({dt:.1f} s)"}


def run_ours(a, rank: int, world: int, local_rank: int) -> None:
    import torch
    import simba_b200 as S

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    inst = make_workload(1 + rank, 64)
    L = a.sweep
    cand_step = sweep_candidates(inst.num_variables, 2, L)
    stream = torch.cuda.Stream()
    sess = S.Session(inst, device=local_rank, stream=stream.cuda_stream)
    with torch.cuda.stream(stream):
        for _ in range(max(a.warmup, 3)):
            r = sess.sweep(2, L)
            assert r.status == S.NOT_FOUND and r.candidates == cand_step, r
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        clocks = Clocks(local_rank)
        clocks.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        kernel_ms, alg_ops, launches, evaluated = 0.0, 0, 0, 0
        for _ in range(a.steps):
            r = sess.sweep(2, L)
            kernel_ms += r.kernel_ms
            alg_ops += r.alg_ops
            launches += r.launches
            evaluated += r.evaluated
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    total_cand = cand_step * a.steps * world
    value = total_cand / (ms / 1e3)

    # end to end through the public C ABI from host buffers
    e2e = None
    if not a.no_e2e:
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        S.solve(inst, L + 1, device=local_rank)  # warm-up: module loading, allocator
        times = []
        for i in range(max(1, min(a.steps, 3))):
            t0 = time.perf_counter()
            rr = S.solve(inst, L + 1, device=local_rank)
            times.append(time.perf_counter() - t0)
            assert rr.status == S.NOT_FOUND and rr.candidates == cand_step
        el = statistics.mean(times)
        if dist:
            t = torch.tensor([el], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        h2d = (inst.num_examples * inst.num_variables + inst.num_examples) * 8
        e2e = {"value": cand_step * world / el, "unit": "candidate-evals/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 64 * (L - 1),
               "seconds_per_step": el}

    if rank == 0:
        peak = S.int_peak(local_rank)
        alu_peak = S.alu_peak(local_rank)
        kernel_s = kernel_ms / 1e3
        achieved = alg_ops / kernel_s if kernel_s > 0 else 0.0
        traffic = None
        prof = ROOT / "profiles" / "spine_kernel_size12_u64_full.md"
        if prof.exists():
            import re
            m = re.search(r"\|\s*dram_bytes_per_candidate\s*\|\s*([0-9.eE+-]+)", prof.read_text())
            if m:
                # DRAM bytes per candidate from the ncu capture, times the
                # candidates of one average spine-kernel launch
                traffic = float(m.group(1)) * evaluated / max(1, a.steps * (L - 1))
        out = {
            "metric": "candidate-evals/s", "value": value, "unit": "candidate-evals/s",
            "n_gpus": world, "steps": a.steps, "warmup": max(a.warmup, 3),
            "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": f"plain-search sweep of sizes 2..{L}: {N_VARS} vars + const 1 "
                                   f"(4 terminals), {N_SAMPLES} uint64 samples, SplitMix64 seed 1+rank, "
                                   "unsatisfiable target (the size-15 config with its outputs "
                                   "randomised so every block is searched)",
                       "candidates_per_step": cand_step, "engine": "tabled spine kernel",
                       "l2": "inputs larger than L2 (value tables of 4 samples up to 5.8 GB)",
                       "parallelism": f"independent instances x{world}"},
            "e2e": e2e,
            "roofline": {"bound": "int-alu", "achieved": achieved / 1e12, "peak": peak / 1e12,
                         "unit": "Tlane-ops/s", "frac": achieved / peak if peak else None,
                         "traffic": traffic,
                         "kernel": "spine_kernel", "kernel_ms_per_step": kernel_ms / a.steps,
                         "alg_ops_per_candidate": alg_ops / max(1, evaluated),
                         "peak_source": "measured live: simba_int_peak (LOP3+IMAD chains)",
                         "alu_pipe_peak": alu_peak / 1e12,
                         "frac_of_alu_pipe": achieved / alu_peak if alu_peak else None},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if not a.no_cpu:
            try:
                out["cpu_baseline"] = cpu_baseline(inst, L)
            except Exception as e:  # the oracle is optional on the GPU box
                out["cpu_baseline"] = {"value": None, "error": str(e)}
        print(json.dumps(out), flush=True)
    del sess
    if dist:
        dist.destroy_process_group()


def run_reference(a, rank: int) -> None:
    """The reference's own CUDA build on the uint32 version of the workload."""
    if rank != 0:
        return
    exe = ROOT / "oracle" / "_ref" / "simba_nocache"  # built by __graft_entry__.build()
    inst = make_workload(1, 32)
    L = REF_L
    cand = sweep_candidates(inst.num_variables, 2, L)
    cfg = {"workload": f"plain-search sweep of sizes 2..{L}: {N_VARS} vars + const 1, {N_SAMPLES} "
                       "samples, unsatisfiable target; uint32 (the reference has no uint64 path)",
           "candidates_per_step": cand}
    if not exe.exists():
        print(json.dumps({"impl": "reference", "unavailable": "reference executable not built "
                          "(oracle/_ref/simba_nocache missing)"}))
        return
    with tempfile.TemporaryDirectory() as td:
        p = Path(td) / "sweep.json"
        inst.write(p)

        def once(max_len: int) -> float:
            r = subprocess.run([str(exe), str(p), str(max_len)], capture_output=True, text=True,
                               timeout=600)
            line = r.stdout.strip().splitlines()[-1]
            return float(line.rsplit(",", 1)[1])

        init = statistics.median([once(2) for _ in range(max(a.warmup, 3))])
        for _ in range(1):
            once(L + 1)
        steps = [once(L + 1) for _ in range(a.steps)]
    search = [max(t - init, 1e-9) for t in steps]
    value = cand / statistics.mean(search)
    out = {"impl": "reference", "metric": "candidate-evals/s", "value": value,
           "unit": "candidate-evals/s", "n_gpus": 1, "steps": a.steps, "warmup": max(a.warmup, 3),
           "ms_per_step": statistics.mean(search) * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
           "config": cfg,
           "cpu_baseline": {"kind": "reference", "value": value, "unit": "candidate-evals/s",
                            "cores": 1, "sample": f"reference CUDA executable rebuilt for sm_100a "
                            f"(GPU; 1 host thread), sizes 2..{L}; its own timer minus the "
                            f"{init:.3f} s CUDA start-up measured with maxLen 2"},
           "e2e": {"value": value, "unit": "candidate-evals/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0},
           "reference_seconds_per_step_incl_context": statistics.mean(steps)}
    print(json.dumps(out), flush=True)


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.case:
        run_case(a.case)
        return
    if a.impl == "reference":
        run_reference(a, rank)
        return
    run_ours(a, rank, world, local)


if __name__ == "__main__":
    main()
