#!/usr/bin/env python
"""Benchmark of the statevector circuit-run path on B200.

Default workload (one step = one full circuit run):
  30-qubit random brickwork circuit, depth 40 (1200 U3 + 580 CNOT = 1780 gates),
  complex64 state (8 GiB, larger than L2 -> no flush needed), |0..0> reset,
  the circuit run by the tensor pass engine (per HBM pass up to three fused
  5-qubit unitaries as split-FP16 tcgen05 GEMMs), then all <Z_i> (FP64).
  metric = gates/s (original gates per second, whole job over all ranks).

Also reported (one untimed run each): the complex128 run of the same circuit
and 1-F / max|d<Z_i>| of complex64 against it and against the complex128
per-gate path; the unfused tiled engine (every gate applied on its own to a
shared-memory tile) and the plain per-gate path (one kernel launch per gate)
with their times and algorithmic HBM GB/s.

  python bench.py [--gpus N --steps K --warmup W]     engine arm
  python bench.py --impl reference                   CPU reference arm (oracle port)

Multi-GPU: the path does not shard (one state per GPU), so N ranks run N
independent replicas ("weak" scaling); value = all ranks' gates / max time.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

HBM_FALLBACK_GBS = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


class ClockSampler:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        self.file.flush()
        rows = []
        for line in Path(self.file.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            if self.uuid and self.uuid not in parts[0]:
                continue
            rows.append(parts)
        os.unlink(self.file.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_reference_rate(gates, n, f32, budget_s, threads=0):
    """Oracle (CPU restatement of the reference path) gates/s on a bounded
    prefix of the circuit: gates are applied one by one until `budget_s`."""
    from oracle import oracle as O
    if threads:
        O.set_threads(threads)
    st = O.OracleState(n, f32=f32)
    done, t0 = 0, time.perf_counter()
    while done < len(gates) and time.perf_counter() - t0 < budget_s:
        st.apply([gates[done]])
        done += 1
    el = time.perf_counter() - t0
    return done / el, done, el, O.max_threads()


def cpu_circuit_rate(items, budget_s, read):
    """Oracle circuits/s over a stride sample of (n, gates) items: circuits are
    taken at a fixed stride through the list (every size class appears) and run
    one by one, gates then the read-out `read(state, k)`, until `budget_s`; a
    circuit cut off by the budget counts by the fraction of its gates done."""
    from oracle import oracle as O
    stride = max(1, len(items) // 64)
    order = [i for s0 in range(stride) for i in range(s0, len(items), stride)]
    done, t0 = 0.0, time.perf_counter()
    for i in order:
        if time.perf_counter() - t0 >= budget_s:
            break
        n, gates = items[i]
        st = O.OracleState(n, f32=True)
        g = 0
        while g < len(gates) and time.perf_counter() - t0 < budget_s:
            st.apply(gates[g:g + 8])
            g += 8
        if g < len(gates):
            done += g / len(gates)
            break
        read(st, i)
        done += 1
    el = time.perf_counter() - t0
    return done / el, done, el, O.max_threads(), stride


def run_reference(args):
    from nqpu_b200.circuits import brickwork
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n, depth = args.qubits, args.depth
    gates = brickwork(n, depth, args.seed)
    f32 = args.dtype == "c64"
    # warm-up: untimed gate applications (page the 8-16 GiB host state in)
    from oracle import oracle as O
    st = O.OracleState(n, f32=f32)
    for i in range(args.warmup):
        st.apply([gates[i % len(gates)]])
    # each step applies a bounded slice of the circuit (~`--ref-step-s` seconds)
    t0 = time.perf_counter()
    st.apply([gates[0]])
    per_gate = time.perf_counter() - t0
    g_step = max(1, int(args.ref_step_s / max(per_gate, 1e-6)))
    times, cnt, pos = [], 0, 1
    for _ in range(args.steps):
        sl = [gates[(pos + j) % len(gates)] for j in range(g_step)]
        t0 = time.perf_counter()
        st.apply(sl)
        times.append(time.perf_counter() - t0)
        cnt += g_step
        pos += g_step
    el = sum(times)
    value = cnt / el
    cores = O.max_threads()
    line = {
        "impl": "reference", "metric": f"gates/s ({n}q {'complex64' if f32 else 'complex128'} brickwork)",
        "value": value,
        "unit": "gates/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "c64" if f32 else "c128", "data": "synthetic",
        "config": {"workload": f"brickwork {n}q depth {depth} {'complex64' if f32 else 'complex128'}",
                   "gates": len(gates), "seed": args.seed},
        "cpu_baseline": {"value": value, "unit": "gates/s", "cores": cores, "kind": "port",
                         "sample": f"{g_step} gates per step x {args.steps} steps of the {n}q circuit, "
                                   f"per-gate full passes, OpenMP {cores} threads"},
        "e2e": {"value": value, "unit": "gates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# DRAM bytes per amplitude per launch of the dominant kernels, from ncu
# captures (dram__bytes_read.sum + dram__bytes_write.sum of one launch divided
# by the amplitudes it covers) on 26-qubit complex64 cases; a full-size launch
# moves the same bytes per amplitude (every amplitude is read and written once
# per pass), so the per-launch traffic is this figure times 2^n.
DRAM_BYTES_PER_AMP = {
    "k_tile_pass": 15.14,  # 26q brickwork depth 8, two launches averaged
    "k_tc_pass": 15.12,    # 26q brickwork depth 10, two launches averaged (537.0 MB read + 477.4 MB written)
}


MODE_DESCRIPTIONS = {
    "tensor": "per HBM pass, up to 3 fused 5-qubit unitaries (32x32 complex, every original gate "
              "folded in) as tcgen05 GEMMs on split-FP16 operands with FP32 accumulation",
    "tiled": "per HBM pass, every gate applied on its own (unfused) to a 2^12-amplitude shared-memory tile, "
             "SIMT FP32/FP64",
    "pergate": "one kernel per gate over the whole state",
    "fused": "one 5-qubit fused unitary per launch, split-TF32 tcgen05 GEMM",
}


def tc_pass_flops(unitaries, n):
    """Tensor-core FLOPs of the tensor pass mode: every fused unitary runs, on
    each 2^12-amplitude tile, A_hi B_hi^T, A_hi B_lo^T and A_lo B_hi^T (three
    128 x 64 x 64 products)."""
    return unitaries * (1 << (n - 12)) * 3 * 2 * 128 * 64 * 64


def tensor_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        return float(json.loads(p.read_text())["bf16_tflops"])
    return 1590.0


def traffic_per_launch(kernel, n):
    b = DRAM_BYTES_PER_AMP.get(kernel)
    return None if b is None else b * (1 << n)


def run_engine(args):
    import torch

    from nqpu_b200 import replicas
    rank, local, world = replicas.world()
    if world > 1:
        torch.cuda.set_device(local)
    replicas.init("nccl", timeout_s=300)
    dev = torch.device("cuda", local if world > 1 else 0)
    torch.cuda.set_device(dev)

    from nqpu_b200 import _lib
    from nqpu_b200.circuits import brickwork
    from nqpu_b200.state import Circuit, StateVector, MODES
    lib = _lib.load()

    n, depth = args.qubits, args.depth
    if args.tile_ctas:
        _lib.check(lib.nqpu_tile_config_set(1 if args.dtype == "c64" else 0, args.tile_ctas), "tile_config")
    if args.circuit == "qft":
        from nqpu_b200.circuits import qft
        gates = qft(n)
    else:
        gates = brickwork(n, depth, args.seed)
    G = len(gates)
    amp_bytes = 8 if args.dtype == "c64" else 16
    S = (1 << n) * amp_bytes
    circ = Circuit(n, gates)
    if args.mode == "auto":
        # the engine's own choice (NQPU_MODE_AUTO), timed as the mode it picks
        am = C.c_int(-1)
        _lib.check(lib.nqpu_circuit_auto_mode(circ.h_, n, 1 if args.dtype == "c64" else 0, C.byref(am)), "auto_mode")
        args.mode = {v: k for k, v in MODES.items()}[am.value]
        args.auto = True
    stats = circ.plan_stats(n, args.dtype, args.mode)
    sv = StateVector(n, args.dtype)
    stream = torch.cuda.ExternalStream(lib.nqpu_state_cuda_stream(sv.h_), device=dev)
    zout = np.empty(n, dtype=np.float64)
    zptr = zout.ctypes.data_as(C.POINTER(C.c_double))
    maxl = 4096
    lms = (C.c_float * maxl)()
    cnt = C.c_uint32()

    def step(profile=False):
        _lib.check(lib.nqpu_state_reset(sv.h_), "reset")
        if profile:
            _lib.check(lib.nqpu_circuit_profile(circ.h_, sv.h_, MODES[args.mode], lms, maxl, C.byref(cnt)), "profile")
        else:
            _lib.check(lib.nqpu_circuit_execute_ex(circ.h_, sv.h_, MODES[args.mode]), "execute")
        _lib.check(lib.nqpu_expectation_z_all(sv.h_, zptr, n), "zall")

    for _ in range(args.warmup):
        step()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    replicas.barrier()
    torch.cuda.synchronize(dev)
    sv.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    launch_ms = []
    for _ in range(args.steps):
        step(profile=True)
        launch_ms.extend(lms[i] for i in range(cnt.value))
    ev1.record(stream)
    ev1.synchronize()
    sv.synchronize()
    torch.cuda.synchronize(dev)
    replicas.barrier()
    clk = clocks.stop()
    # whole-job rate: every rank ran G * steps gates; time = max over ranks
    value, el_s = replicas.replica_rate(G * args.steps, ev0.elapsed_time(ev1) / 1000.0, device=dev)
    el_ms = el_s * 1000.0
    z_c64 = zout.copy()

    # roofline of the dominant kernel (the tiled pass): 2S algorithmic bytes per launch
    peak, peak_kind = peaks()
    avg_launch_ms = float(np.mean(launch_ms)) if launch_ms else float("nan")
    achieved = 2 * S / (avg_launch_ms / 1000.0) / 1e9
    kernel = {"tiled": "k_tile_pass", "tensor": "k_tc_pass", "fused": "k_fused_apply",
              "pergate": "k_pg_*"}[args.mode]
    traffic = traffic_per_launch(kernel, n) if args.dtype == "c64" else None
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                "traffic": traffic, "traffic_source": "ncu DRAM bytes per amplitude of a 26-qubit capture x 2^n",
                "algorithmic_bytes_per_launch": 2 * S,
                "launches_per_step": stats["passes"], "avg_launch_ms": avg_launch_ms,
                "pass_time_share": (sum(launch_ms) / el_ms) if el_ms else None}
    mhz = (clk or {}).get("sm_mhz") or 1965.0
    pass_s = sum(launch_ms) / 1000.0 if launch_ms else float("nan")
    if args.mode == "tensor":
        # tensor-pipe work of the pass kernel: per tile (2^12 amplitudes) and
        # fused unitary, three 128 x 64 x 64 FP16 GEMMs
        fl = tc_pass_flops(stats["stages"], n) * args.steps
        roofline["tensor"] = {"achieved_tflops": fl / pass_s / 1e12, "peak_tflops": tensor_peak(),
                              "frac": fl / pass_s / 1e12 / tensor_peak(), "flops_per_step": fl // args.steps,
                              "peak_kind": "measured dense bf16 (cuBLAS burst); FP16 runs at the same rate"}
    elif args.mode == "tiled":
        # the tiled pass is bound by arithmetic issue, not HBM: its rate against the
        # FP32 peak (148 SMs x 128 lanes x 2 flops per cycle at the sampled clock) for
        # complex64, the FP64 peak (148 SMs x 64 lanes x 2) for complex128
        from nqpu_b200.circuits import algorithmic_flops
        lanes = 128 if args.dtype == "c64" else 64
        arith_peak = 148 * lanes * 2 * mhz * 1e6 / 1e12
        fl = algorithmic_flops(gates, n) * args.steps
        roofline["fp32" if args.dtype == "c64" else "fp64"] = {
            "achieved_tflops": fl / pass_s / 1e12, "peak_tflops": arith_peak,
            "frac": fl / pass_s / 1e12 / arith_peak, "flops_per_step": fl // args.steps,
            "peak_kind": "nominal at the sampled SM clock"}
    launches_per_step = stats["passes"] + 1 + 2  # passes + reset + zsums (2 kernels)

    extra = {}
    if rank == 0 and world == 1 and not args.quick:
        # accuracy: complex64 against the complex128 (FP64) run of the same circuit
        ref_dtype = "c128" if args.dtype == "c64" else None
        if ref_dtype:
            sv128 = StateVector(n, ref_dtype)
            mode128 = "tiled" if args.mode in ("tensor", "fused") else args.mode  # complex64-only modes
            t0 = time.perf_counter()
            circ.execute(sv128, mode128)
            z128 = sv128.expectation_z_all()
            t128 = time.perf_counter() - t0
            f = sv.fidelity(sv128)
            extra["accuracy_vs_fp64"] = {"one_minus_F": 1.0 - f, "max_abs_dZ": float(np.abs(z_c64 - z128).max()),
                                         "tolerance": {"one_minus_F": 1e-5, "max_abs_dZ": 1e-5}}
            from nqpu_b200.circuits import algorithmic_flops
            fl64 = algorithmic_flops(gates, n)
            mhz64 = (clk or {}).get("sm_mhz") or 1965.0
            # FP64 peak of the SIMT pipes: 148 SMs x 64 FP64 FMA lanes x 2 flops per cycle
            fp64_peak = 148 * 64 * 2 * mhz64 * 1e6 / 1e12
            passes128 = circ.plan_stats(n, "c128", mode128)["passes"]
            extra["complex128_run"] = {
                "gates_per_s": G / t128, "seconds": t128, "mode": mode128, "passes": passes128,
                "hbm_GBps": passes128 * 2 * (1 << n) * 16 / t128 / 1e9,
                "hbm_frac": passes128 * 2 * (1 << n) * 16 / t128 / 1e9 / peak,
                "fp64": {"achieved_tflops": fl64 / t128 / 1e12, "peak_tflops": fp64_peak,
                         "frac": fl64 / t128 / 1e12 / fp64_peak, "flops": fl64,
                         "peak_kind": "nominal FP64 SIMT rate at the sampled SM clock"}}
            # the same circuit through the per-gate path in complex128 (one
            # kernel per gate, no planner): a check of the planned engine at
            # the full size that does not rest on the planner
            svpg = StateVector(n, "c128")
            circ.execute(svpg, "pergate")
            zpg = svpg.expectation_z_all()
            extra["accuracy_vs_pergate"] = {
                "reference": "complex128 per-gate path (one kernel per gate, no tiled plan)",
                f"{args.mode}_c64": {"one_minus_F": 1.0 - sv.fidelity(svpg),
                                     "max_abs_dZ": float(np.abs(z_c64 - zpg).max())},
                f"{mode128}_c128": {"one_minus_F": 1.0 - sv128.fidelity(svpg),
                                    "max_abs_dZ": float(np.abs(z128 - zpg).max())},
                "tolerance": {"c64": 1e-5, "c128": 1e-12}}
            svpg.close()
            sv128.close()
        # plain per-gate path: one launch per gate, algorithmic GB/s
        pg_ms = (C.c_float * maxl)()
        pcnt = C.c_uint32()
        _lib.check(lib.nqpu_state_reset(sv.h_), "reset")
        lib.nqpu_circuit_execute_ex(circ.h_, sv.h_, MODES["pergate"])  # warm
        _lib.check(lib.nqpu_state_reset(sv.h_), "reset")
        _lib.check(lib.nqpu_circuit_profile(circ.h_, sv.h_, MODES["pergate"], pg_ms, maxl, C.byref(pcnt)), "profile")
        from nqpu_b200.circuits import algorithmic_bytes
        tot_ms = sum(pg_ms[i] for i in range(pcnt.value))
        u3_ms = [pg_ms[i] for i in range(pcnt.value) if gates[i][0] == "u3"]
        cx_ms = [pg_ms[i] for i in range(pcnt.value) if gates[i][0] == "cx"]
        extra["pergate_path"] = {
            "gates_per_s": G / (tot_ms / 1000), "seconds": tot_ms / 1000,
            "algorithmic_GBps": algorithmic_bytes(gates, n, amp_bytes) / (tot_ms / 1000) / 1e9,
            "u3_GBps": 2 * S / (np.mean(u3_ms) / 1000) / 1e9 if u3_ms else None,
            "cnot_GBps": S / (np.mean(cx_ms) / 1000) / 1e9 if cx_ms else None,
            "frac_of_peak": algorithmic_bytes(gates, n, amp_bytes) / (tot_ms / 1000) / 1e9 / peak,
        }
        if args.mode != "tiled":
            # the unfused tiled engine on the same circuit: every gate applied
            # on its own to the shared-memory tile (SIMT FP32), several per pass
            tl_ms = (C.c_float * maxl)()
            tcnt = C.c_uint32()
            _lib.check(lib.nqpu_state_reset(sv.h_), "reset")
            _lib.check(lib.nqpu_circuit_execute_ex(circ.h_, sv.h_, MODES["tiled"]), "execute")  # warm
            _lib.check(lib.nqpu_state_reset(sv.h_), "reset")
            _lib.check(lib.nqpu_circuit_profile(circ.h_, sv.h_, MODES["tiled"], tl_ms, maxl, C.byref(tcnt)),
                       "profile")
            tms = [tl_ms[i] for i in range(tcnt.value)]
            extra["tiled_path"] = {
                "gates_per_s": G / (sum(tms) / 1000), "seconds": sum(tms) / 1000, "passes": len(tms),
                "kernel": "k_tile_pass", "avg_launch_ms": float(np.mean(tms)),
                "frac_of_peak": 2 * S / (np.mean(tms) / 1000) / 1e9 / peak,
                "timing": "CUDA events around each pass launch, one run after a warm-up run"}

    # e2e: host gate list -> circuit handle -> execute (plan build + H2D) -> <Z_i> D2H
    e2e = None
    if not args.quick:
        torch.cuda.synchronize(dev)
        h2d = stats.get("upload_bytes", 0)
        t_e2e = []
        for _ in range(max(1, args.e2e_steps)):
            t0 = time.perf_counter()
            c2 = Circuit(n, gates)
            _lib.check(lib.nqpu_state_reset(sv.h_), "reset")
            e2e_mode = MODES["auto"] if getattr(args, "auto", False) else MODES[args.mode]
            _lib.check(lib.nqpu_circuit_execute_ex(c2.h_, sv.h_, e2e_mode), "execute")
            _lib.check(lib.nqpu_expectation_z_all(sv.h_, zptr, n), "zall")
            t_e2e.append(time.perf_counter() - t0)
            c2.close()
        et = replicas.max_over_ranks(float(np.mean(t_e2e)), device=dev)
        e2e = {"value": G * world / et, "unit": "gates/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": 8 * n, "seconds_per_step": et,
               "timing": "host wall clock around create+execute+reduce (includes the mode choice and plan build)"}

    cpu = None
    if rank == 0 and world == 1 and not args.quick and not args.no_cpu:
        rate, done, el, cores = cpu_reference_rate(gates, n, args.dtype == "c64", args.cpu_budget_s)
        cpu = {"value": rate, "unit": "gates/s", "cores": cores, "kind": "port",
               "sample": f"first {done} gates of the {n}q circuit in {el:.1f} s, per-gate full passes"}

    if rank == 0:
        line = {
            "metric": (f"gates/s ({n}q {'complex64' if args.dtype == 'c64' else 'complex128'} brickwork)"
                       if args.circuit == "brickwork"
                       else f"gates/s ({n}q QFT)"), "value": value, "unit": "gates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.dtype, "data": "synthetic",
            "config": {"workload": (f"brickwork {n}q depth {depth}" if args.circuit == "brickwork" else f"QFT {n}q")
                                   + f" {'complex64' if args.dtype == 'c64' else 'complex128'}",
                       "gates": G, "seed": args.seed, "engine_mode": args.mode,
                       "engine_mode_chosen_by": "NQPU_MODE_AUTO" if getattr(args, "auto", False) else "--mode",
                       "engine": MODE_DESCRIPTIONS[args.mode],
                       "plan": {"passes": stats["passes"], "stages": stats["stages"]},
                       "tile_ctas_per_sm": int(lib.nqpu_tile_config_get(1 if args.dtype == "c64" else 0)),
                       "l2": f"state {S / 2**30:.2f} GiB vs 126 MB L2; no flush", "parallelism": f"replicas{world}"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches_per_step * args.steps, "clocks": clk,
        }
        line.update(extra)
    sv.close()
    circ.close()
    if rank == 0 and world == 1 and not args.quick and not args.plain_only:
        # the CPU-runnable configuration and the three forms, each with its own
        # parity, e2e, CPU baseline, roofline and clock record
        line["config1_brickwork20"] = run_config1(args)
        sub = argparse.Namespace(**vars(args))
        sub.qubits = 32
        line["precision"] = run_precision(sub)
        line["batch"] = run_batch(argparse.Namespace(**vars(args)))
        sub = argparse.Namespace(**vars(args))
        sub.rates = args.embedded_rates
        line["serve"] = run_serve(sub)
    if rank == 0:
        print(json.dumps(line), flush=True)
    replicas.shutdown()


def run_config1(args):
    """The CPU-runnable configuration: 20-qubit complex128 brickwork, depth 20,
    seeds 1-3, |0..0>; outputs the final state, all <Z_i> and 1000 shots.  The
    engine's tiled run and the oracle's per-gate passes (the reference's CPU
    path, restated) are both timed in full: 3 warm-up and 5 measured runs per
    seed.  Parity: 1-F, max|amp diff| and max|d<Z_i>| against the oracle, and
    the 1000 shots drawn with the same uniforms."""
    import torch
    from nqpu_b200 import _lib
    from nqpu_b200.circuits import brickwork
    from nqpu_b200.state import Circuit, StateVector, MODES
    from oracle import oracle as O
    lib = _lib.load()
    n, depth, shots = 20, 20, 1000
    out = {"workload": f"brickwork {n}q depth {depth} complex128, seeds 1-3, all <Z_i> + {shots} shots",
           "per_seed": []}
    gpu_s, cpu_s, G_tot = [], [], 0
    for seed in (1, 2, 3):
        gates = brickwork(n, depth, seed)
        G = len(gates)
        G_tot += G
        c = Circuit(n, gates)
        sv = StateVector(n, "c128")
        stream = torch.cuda.ExternalStream(lib.nqpu_state_cuda_stream(sv.h_))
        u = O.xorshift_uniforms(seed, shots)

        def gpu_run():
            sv.reset()
            c.execute(sv, "tiled")
            return sv.expectation_z_all(), sv.sample_with_uniforms(u)
        for _ in range(3):
            gpu_run()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(5):
            z, smp = gpu_run()
        ev1.record(stream)
        ev1.synchronize()
        g_ms = ev0.elapsed_time(ev1) / 5
        amps = sv.amplitudes()

        def cpu_run():
            o = O.OracleState(n)
            o.apply(gates)
            return o, o.expectation_z_all(), o.sample_uniforms(u)
        for _ in range(3):
            cpu_run()
        t0 = time.perf_counter()
        for _ in range(5):
            o, zo, so = cpu_run()
        c_ms = 1000 * (time.perf_counter() - t0) / 5
        ref = o.amplitudes()
        f = abs(np.vdot(ref, amps)) ** 2
        out["per_seed"].append({
            "seed": seed, "gates": G, "gpu_ms": g_ms, "cpu_ms": c_ms,
            "one_minus_F": 1 - f, "max_abs_amp_diff": float(np.abs(amps - ref).max()),
            "max_abs_dZ": float(np.abs(z - zo).max()),
            "shots_equal": int(np.sum(np.asarray(smp) == np.asarray(so))), "shots": shots})
        gpu_s.append(g_ms / 1000)
        cpu_s.append(c_ms / 1000)
        sv.close()
        c.close()
    out["gpu_gates_per_s"] = G_tot / sum(gpu_s)
    out["cpu_baseline"] = {"value": G_tot / sum(cpu_s), "unit": "gates/s", "cores": O.max_threads(),
                           "kind": "port", "sample": "the full circuit of each seed, 3 warm-up + 5 timed runs, "
                                                     "per-gate passes + all <Z_i> + 1000 shots"}
    out["speedup_vs_cpu"] = out["gpu_gates_per_s"] / out["cpu_baseline"]["value"]
    out["tolerance"] = {"one_minus_F": 1e-12, "max_abs_amp_diff": 1e-12, "max_abs_dZ": 1e-12,
                        "shots": "equal up to CDF summation ties"}
    out["timing"] = "gpu: CUDA events on the state's stream around 5 runs (reset, tiled circuit, all <Z_i>, " \
                    "1000 shots with host read-back); cpu: wall clock around 5 oracle runs"
    return out


def run_precision(args):
    """Precision form: 32-qubit first-order Trotterised TFIM (open chain, J = 1,
    h_i ~ U[0.6, 1.0], dt = 0.05, 100 steps; RZZ(2 J dt) on every bond then
    RX(2 h_i dt) on every site) from the Neel state |0101...>, complex64 state,
    gates fused into 5-qubit unitaries applied as split-TF32 tcgen05 GEMMs.
    <Z_i> and <Z0 Z1> every 10 steps, with errors against the FP64 run
    (complex128, unfused tiled engine) of the same circuit."""
    import torch
    from nqpu_b200 import _lib
    from nqpu_b200.circuits import neel_index, tfim_trotter
    from nqpu_b200.state import Circuit, StateVector, MODES
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n, steps, every = args.qubits, args.tfim_steps, 10
    chunk, h = tfim_trotter(n, every, seed=args.seed)
    c = Circuit(n, chunk)
    zz = "ZZ" + "I" * (n - 2)
    maxl = 8192
    lms = (C.c_float * maxl)()
    cnt = C.c_uint32()

    def run(dtype, mode):
        sv = StateVector(n, dtype)
        sv.set_basis(neel_index(n))
        rec, launches = [], []
        for _ in range(steps // every):
            _lib.check(lib.nqpu_circuit_profile(c.h_, sv.h_, MODES[mode], lms, maxl, C.byref(cnt)), "profile")
            launches.extend(lms[i] for i in range(cnt.value))
            rec.append((sv.expectation_z_all(), sv.expectation_pauli_string(zz)))
        return sv, rec, launches

    # warm-up (plans, module load)
    w = StateVector(n, "c64")
    c.execute(w, "fused")
    w.close()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    sv64, rec64, l64 = run("c64", "fused")
    clk = clocks.stop()
    sv128, rec128, l128 = run("c128", "tiled")
    f = sv64.fidelity(sv128)

    def checkpoints(rec):
        return [{"step": every * (i + 1), "max_abs_dZ": float(np.abs(a[0] - b[0]).max()), "abs_dZ0Z1": abs(a[1] - b[1])}
                for i, (a, b) in enumerate(zip(rec, rec128))]

    errs = checkpoints(rec64)
    # the same circuit through the tensor-core pass mode (several fused
    # unitaries per HBM pass, split FP16) and the engine's own mode choice
    am = C.c_int(-1)
    _lib.check(lib.nqpu_circuit_auto_mode(c.h_, n, 1, C.byref(am)), "auto_mode")
    tensor = None
    if not args.quick:
        w = StateVector(n, "c64")
        c.execute(w, "tensor")  # plan and module load
        w.close()
        sv_tc, rec_tc, l_tc = run("c64", "tensor")
        e_tc = checkpoints(rec_tc)
        st_tc = c.plan_stats(n, "c64", "tensor")
        tensor = {"gates_per_s": len(chunk) * (steps // every) / (sum(l_tc) / 1000), "seconds": sum(l_tc) / 1000,
                  "launches": len(l_tc), "kernel": "k_tc_pass",
                  "fused_unitaries": st_tc["stages"] * (steps // every),
                  "hbm_frac": 2 * (1 << n) * 8 / (np.mean(l_tc) / 1000) / 1e9 / peaks()[0],
                  "accuracy_vs_fp64": {"one_minus_F": 1 - sv_tc.fidelity(sv128),
                                       "max_abs_dZ": max(e["max_abs_dZ"] for e in e_tc),
                                       "max_abs_dZ0Z1": max(e["abs_dZ0Z1"] for e in e_tc)},
                  "engine": MODE_DESCRIPTIONS["tensor"]}
        sv_tc.close()
    sv128.close()
    plain = None
    if not args.quick:
        sv_t, rec_t, l_t = run("c64", "tiled")
        plain = {"gates_per_s": len(chunk) * (steps // every) / (sum(l_t) / 1000), "seconds": sum(l_t) / 1000,
                 "launches": len(l_t)}
        sv_t.close()
    sv64.close()
    peak, peak_kind = peaks()
    S = (1 << n) * 8
    fused_ms = sum(l64)
    G = len(chunk) * (steps // every)
    st = c.plan_stats(n, "c64", "fused")
    # e2e through the public API: gate list -> circuit -> fused runs with the
    # <Z_i> and <Z0 Z1> read-outs on the host, wall clock
    e2e = None
    if not args.quick:
        t0 = time.perf_counter()
        ce = Circuit(n, chunk)
        se = StateVector(n, "c64")
        se.set_basis(neel_index(n))
        for _ in range(steps // every):
            ce.execute(se, "fused")
            se.expectation_z_all()
            se.expectation_pauli_string(zz)
        et = time.perf_counter() - t0
        se.close()
        ce.close()
        e2e = {"value": G / et, "unit": "gates/s", "h2d_bytes_per_step": int(st.get("upload_bytes", 0)),
               "d2h_bytes_per_step": (8 * n + 8) * (steps // every), "seconds_per_step": et,
               "timing": "host wall clock: circuit from the gate list, state init, fused runs (plan build and "
                         "B-operand upload included) and the read-outs every 10 steps"}
    # CPU baseline: the oracle's per-gate passes on the same TFIM chunk at a
    # size whose complex64 state fits host memory comfortably (26 qubits),
    # scaled to 32 qubits by the state size (each pass is linear in 2^n)
    cpu = None
    if not args.quick and not args.no_cpu:
        nc = min(n, 26)
        cg, _ = tfim_trotter(nc, every, seed=args.seed)
        rate, done, el, cores = cpu_reference_rate(cg, nc, True, args.cpu_budget_s)
        cpu = {"value": rate / (1 << (n - nc)), "unit": "gates/s", "cores": cores, "kind": "port",
               "sample": f"first {done} gates of the {nc}-qubit TFIM chunk in {el:.1f} s ({rate:.1f} gates/s), "
                         f"scaled by 2^{nc - n} to {n} qubits"}
    line = {
        "form": "precision", "metric": f"gates/s ({n}q TFIM Trotter, fused split-TF32 tensor cores)",
        "value": G / (fused_ms / 1000), "unit": "gates/s", "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": fused_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": "synthetic",
        "config": {"workload": f"TFIM {n}q {steps} Trotter steps dt 0.05, Neel start", "gates": G,
                   "fused_unitaries": st["passes"] * (steps // every), "seed": args.seed},
        "seconds": fused_ms / 1000,
        "roofline": {"bound": "hbm", "kernel": "k_fused_apply", "achieved": 2 * S / (np.mean(l64) / 1000) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": 2 * S / (np.mean(l64) / 1000) / 1e9 / peak,
                     "peak_kind": peak_kind, "avg_launch_ms": float(np.mean(l64)),
                     "tensor_tflops": 24 * 2 * 128 * 64 * 8 * ((1 << n) // 4096) / (np.mean(l64) / 1000) / 1e12},
        "accuracy_vs_fp64": {"one_minus_F": 1 - f, "checkpoints": errs,
                             "max_abs_dZ": max(e["max_abs_dZ"] for e in errs),
                             "max_abs_dZ0Z1": max(e["abs_dZ0Z1"] for e in errs)},
        "fp64_reference_seconds": sum(l128) / 1000, "plain_tiled_c64": plain,
        "tensor_pass_c64": tensor, "auto_mode_choice": {0: "tiled", 3: "tensor"}.get(am.value, am.value),
        "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": len(l64), "clocks": clk,
    }
    return line


def run_batch(args):
    """Batching form: 4096 hardware-efficient-ansatz circuits (n ~ U{10..22},
    L ~ U{2..12} layers of RY RZ on every qubit + CZ ladder, angles U[0, 2pi)),
    each returning <H> of its own Ising chain H = sum J_i Z_i Z_{i+1} + sum h_i X_i
    (J, h ~ U[-1, 1]); complex64 states, FP64 reductions, one persistent
    graph-captured launch per step with the autotuner's configuration.
    Compared with the plain per-circuit path (one kernel per gate, then the
    Pauli-sum expectation, one circuit after another) on a stratified sample."""
    import torch
    from nqpu_b200 import autotune
    from nqpu_b200.batch import Batch, ising_terms
    from nqpu_b200.circuits import hea_batch
    from nqpu_b200.state import Circuit, StateVector
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    count = args.circuits
    items = hea_batch(count, args.seed, nmin=10, nmax=22, lmin=2, lmax=12)
    # the same circuits as flat gate arrays (the input of Circuit.from_arrays)
    arrs = hea_batch(count, args.seed, nmin=10, nmax=22, lmin=2, lmax=12, arrays=True)
    G = sum(len(g) for _, g, _, _ in items)
    t0 = time.perf_counter()
    circs = [Circuit.from_arrays(n, *a) for n, a, _, _ in arrs]
    host_build_s = time.perf_counter() - t0
    log = (lambda m: print(m, file=sys.stderr, flush=True)) if args.verbose else None
    if args.quick:  # timed region only: library defaults, no tuning
        cfg, tune_report = dict(autotune.DEFAULT), {"skipped": "--quick"}
    else:
        cfg, tune_report = autotune.tune(items, sample_size=min(args.tune_sample, count), circuits=circs,
                                         use_cache=not args.no_tune_cache, log=log)
    b = Batch()
    b.config(**cfg)
    for c, (n, g, J, h) in zip(circs, items):
        b.add_ising(c, J, h)
    t0 = time.perf_counter()
    b.prepare()
    prepare_s = time.perf_counter() - t0
    st = b.stats()
    for _ in range(args.warmup):
        res = b.run()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    clocks.start()
    torch.cuda.synchronize(dev)
    dev_ms, wall = [], time.perf_counter()
    steps = max(args.steps, 10)  # one step is ~0.1 s: time at least ten replays
    for _ in range(steps):
        res = b.run()
        dev_ms.append(b.last_run_ms())
    wall = time.perf_counter() - wall
    clk = clocks.stop()
    tot_ms = float(sum(dev_ms))
    value = count * steps / (tot_ms / 1000)

    # the HBM-resident part of the work: 2S per pass tile sweep + S for <H>, S = 2^n * 8
    big_bytes = 0
    sample = autotune.stratified_sample(items, 0 if args.quick else min(args.plain_sample, count))
    for i in range(count):
        n = items[i][0]
        if n > cfg["small_max_qubits"]:
            p = circs[i].plan_stats(n, "c64", "tiled")["passes"]
            big_bytes += (2 * p + 1) * (1 << n) * 8
    peak, peak_kind = peaks()
    achieved = big_bytes / (np.mean(dev_ms) / 1000) / 1e9

    # plain per-circuit path and per-circuit tiled path on a stratified sample;
    # accuracy of the batch against the FP64 (complex128) per-circuit run
    states = {}
    plain_s = tiled_s = 0.0
    err_plain = err_fp64 = 0.0
    for i in sample:
        n, g, J, h = items[i]
        terms = ising_terms(n, J, h)
        scale = np.abs(J).sum() + np.abs(h).sum()
        if n not in states:
            states[n] = StateVector(n, "c64")
            circs[i].execute(states[n], "pergate")  # warm the module for this size
        sv = states[n]
        t = time.perf_counter()
        sv.reset()
        circs[i].execute(sv, "pergate")
        e_plain = sv.expectation_pauli_sum(terms)
        plain_s += time.perf_counter() - t
        t = time.perf_counter()
        sv.reset()
        circs[i].execute(sv, "tiled")
        sv.expectation_pauli_sum(terms)
        tiled_s += time.perf_counter() - t
        with StateVector(n, "c128") as s128:
            circs[i].execute(s128, "tiled")
            e64 = s128.expectation_pauli_sum(terms)
        err_plain = max(err_plain, abs(res[i] - e_plain) / scale)
        err_fp64 = max(err_fp64, abs(res[i] - e64) / scale)
    for s in states.values():
        s.close()
    plain_rate = len(sample) / plain_s if sample else None
    tiled_rate = len(sample) / tiled_s if sample else None

    # e2e through the public API: gate arrays -> circuits -> batch -> <H> on the host
    e2e = None
    if not args.quick:
        t = time.perf_counter()
        b2 = Batch()
        b2.config(**cfg)
        t_circ = time.perf_counter()
        b2.add_ising_arrays(arrs)  # every circuit's gate arrays in one call
        t_add = time.perf_counter()
        b2.prepare()
        t_prep = time.perf_counter()
        r2 = b2.run()
        t_run = time.perf_counter()
        et = t_run - t
        assert np.array_equal(r2, res)
        e2e = {"value": count / et, "unit": "circuits/s", "h2d_bytes_per_step": int(st["upload_bytes"]),
               "d2h_bytes_per_step": 8 * count, "seconds_per_step": et,
               "phases_s": {"batch_create": t_circ - t, "batch_add_arrays": t_add - t_circ, "prepare": t_prep - t_add,
                            "run": t_run - t_prep},
               "prepare_phases_s": b2.stats()["prepare_s"],
               "frac_of_device_rate": (count / et) / value,
               "timing": "host wall clock: batch from the circuits' gate arrays (one nqpu_batch_add_ising_arrays "
                         "call), prepare (plans on host threads, uploads, graph capture), one replay, results on the host"}
        b2.close()

    cpu = None
    if not args.quick and not args.no_cpu:
        def read_h(st, i):
            _, _, J, h = items[i]
            n = len(h)
            z = [st.pauli_string("I" * q + "ZZ" + "I" * (n - q - 2)) for q in range(n - 1)]
            x = [st.pauli_string("I" * q + "X" + "I" * (n - q - 1)) for q in range(n)]
            return float(np.dot(J, z) + np.dot(h, x))
        rate, done, el, cores, stride = cpu_circuit_rate([(n, g) for n, g, _, _ in items], args.cpu_budget_s,
                                                         read_h)
        cpu = {"value": rate, "unit": "circuits/s", "cores": cores, "kind": "port",
               "sample": f"{done:.2f} of the {count} circuits (stride {stride}, every size class) in {el:.1f} s: "
                         f"per-gate passes and the Ising <H> Pauli terms"}

    line = {
        "form": "batch", "metric": f"circuits/s ({count} mixed-size HEA circuits, <H> per circuit)",
        "value": value, "unit": "circuits/s", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": tot_ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": "synthetic",
        "config": {"workload": f"{count} HEA circuits n 10-22, 2-12 layers, Ising <H>", "circuits": count,
                   "gates": G, "seed": args.seed, "autotuned": cfg,
                   "small_in_smem": int(st["small"]), "tasks": int(st["tasks"]),
                   "arena_bytes": int(st["arena_bytes"]),
                   "l2": "state arena plus table reads per replay; no flush (work is smem/L2 resident by design)"},
        "autotune": tune_report,
        "roofline": {"bound": "hbm", "kernel": "k_batch", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": big_bytes,
                     "note": "only circuits above the shared-memory threshold move HBM bytes; the rest is "
                             "SM-issue bound in shared memory"},
        "plain_per_circuit_path": {"circuits_per_s": plain_rate, "sample": len(sample),
                                   "what": "per-gate kernels + Pauli-sum <H>, one circuit at a time (host wall)"},
        "tiled_per_circuit_path": {"circuits_per_s": tiled_rate, "sample": len(sample)},
        "speedup_vs_plain": value / plain_rate if plain_rate else None,
        "accuracy": {"max_rel_err_vs_fp64": err_fp64, "max_rel_err_vs_plain_c64": err_plain,
                     "tolerance": "|<H> - <H>_FP64| <= 1e-5 * (sum|J| + sum|h|)"},
        "host_build_s": host_build_s, "prepare_s": prepare_s, "wall_s_timed": wall,
        "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": steps, "clocks": clk,
    }
    b.close()
    return line


def run_serve(args):
    """Serving form: Poisson request streams at swept rates; n = round(exp(U[ln 8,
    ln 28])), brickwork depth ~ U{10..50}, half the requests ask for 1024 shots,
    half for all <Z_i>; admission by an HBM budget of 2^n x 8 B per state with
    states device-resident; latency = submit (before planning) to result ready.
    Compared with the plain per-circuit path (per-gate kernels, one request at a
    time) on a stratified sample of the same requests."""
    import torch
    from nqpu_b200 import autotune
    from nqpu_b200.circuits import brickwork, serving_mix
    from nqpu_b200.server import Server
    from nqpu_b200.state import Circuit, StateVector
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    count = args.requests
    base = serving_mix(count, args.seed, rate=1.0)  # arrival times at 1 req/s; scaled per rate
    t0 = time.perf_counter()
    circs = [Circuit(r["n"], brickwork(r["n"], r["depth"], r["seed"])) for r in base]
    build_s = time.perf_counter() - t0
    G = sum(c.gate_count for c in circs)
    # the server runs each request in NQPU_MODE_AUTO's choice (tensor-core or tiled passes)
    pstats = [c.plan_stats(r["n"], "c64", "auto") for c, r in zip(circs, base)]
    passes = [p_["passes"] for p_ in pstats]
    # bytes each rate step moves: every request's plan tables (and its shot
    # uniforms) host->device, its <Z_i> or outcomes device->host
    h2d_step = sum(int(p_.get("upload_bytes", 0)) + (1024 * 8 if r["kind"] == "shots" else 0)
                   for p_, r in zip(pstats, base))
    d2h_step = sum(8 * r["n"] if r["kind"] == "zall" else 1024 * 8 for r in base)
    launches = sum(1 + p + (2 if r["kind"] == "zall" else 3) for p, r in zip(passes, base))
    budget = int(args.serve_budget_gb * (1 << 30))
    rates = [float(x) for x in args.rates.split(",")]
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass

    srv = Server(hbm_budget_bytes=budget, max_qubits=28, lanes=args.lanes, large_lanes=2, large_qubits=22,
                 max_shots=1024)
    # warm-up: one request of every size class (module load, smem attributes, pool)
    for n in (8, 14, 20, 26):
        c = Circuit(n, brickwork(n, 4, 1))
        rid = srv.submit(c, "zall")
        srv.wait(rid, 60.0)
        srv.result(rid)
        c.close()

    sweep, results_by_rate = [], {}
    clocks = ClockSampler(uuid)
    clocks.start()
    for lam in rates:
        ids = []
        start = time.perf_counter()
        for r, c in zip(base, circs):
            target = start + r["arrival"] / lam
            while True:
                d = target - time.perf_counter()
                if d <= 0:
                    break
                time.sleep(min(d, 0.002))
            ids.append(srv.submit(c, r["kind"], 1024 if r["kind"] == "shots" else 0, r["seed"]))
        srv.wait(0, 600.0)
        span = time.perf_counter() - start
        lat, vals = [], []
        for i in ids:
            v, t = srv.result(i)
            lat.append(t["total_ms"])
            vals.append(v)
        st = srv.stats()
        lat = np.array(lat)
        sweep.append({"rate_per_s": lam, "circuits_per_s": count / span, "p50_ms": float(np.percentile(lat, 50)),
                      "p99_ms": float(np.percentile(lat, 99)), "mean_ms": float(lat.mean()),
                      "makespan_s": span, "peak_concurrent": st["peak_concurrent"],
                      "peak_resident_GB": st["peak_resident_bytes"] / 1e9})
        results_by_rate[lam] = vals
    clk = clocks.stop()
    arena = srv.stats()["arena_bytes"]
    srv.close()
    # identical results at every rate (the mix each request ran in differs)
    same = all(np.array_equal(a, b) for lam in rates[1:] for a, b in zip(results_by_rate[rates[0]],
                                                                         results_by_rate[lam]))

    # plain per-circuit path on a stratified sample; accuracy against complex128
    items = [(r["n"], [None] * r["depth"], None, None) for r in base]
    sample = autotune.stratified_sample(items, min(args.plain_sample, count))
    lib = circs[0].lib
    svc, max_dz, max_inf = [], 0.0, 0.0
    for i in sample:
        r, c = base[i], circs[i]
        with StateVector(r["n"], "c64") as sv:
            c.execute(sv, "pergate")  # warm
            sv.reset()
            t = time.perf_counter()
            c.execute(sv, "pergate")
            if r["kind"] == "zall":
                sv.expectation_z_all()
            else:
                lib.nqpu_set_seed(r["seed"])
                sv.sample(1024)
            svc.append(time.perf_counter() - t)
            if r["n"] <= 26:
                sv.reset()
                c.execute(sv, "auto")  # the server's computation (bitwise, tested)
                with StateVector(r["n"], "c128") as s128:
                    c.execute(s128, "tiled")
                    max_inf = max(max_inf, 1.0 - sv.fidelity(s128))
                    max_dz = max(max_dz, float(np.abs(sv.expectation_z_all() - s128.expectation_z_all()).max()))
    svc = np.array(svc)
    plain_rate = 1.0 / svc.mean()
    top = sweep[-1]
    cpu = None
    if not args.quick and not args.no_cpu:
        from oracle import oracle as O
        def read_req(st, i):
            r = base[i]
            if r["kind"] == "zall":
                return st.expectation_z_all()
            return st.sample_uniforms(O.xorshift_uniforms(r["seed"], 1024))
        reqs = [(r["n"], brickwork(r["n"], r["depth"], r["seed"])) for r in base]
        rate, done, el, cores, stride = cpu_circuit_rate(reqs, args.cpu_budget_s, read_req)
        cpu = {"value": rate, "unit": "circuits/s", "cores": cores, "kind": "port",
               "sample": f"{done:.2f} of the {count} requests (stride {stride}) one after another in {el:.1f} s: "
                         f"per-gate passes, then all <Z_i> or 1024 shots"}
    line = {
        "form": "serve", "metric": "served circuits/s at the highest offered rate (p50/p99 latency beside it)",
        "value": top["circuits_per_s"], "unit": "circuits/s", "n_gpus": 1, "steps": len(rates), "warmup": 4,
        "ms_per_step": 1000 * top["makespan_s"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "c64", "data": "synthetic",
        "config": {"workload": f"{count} Poisson requests per rate, n log-uniform 8-28, brickwork depth 10-50, "
                               "half 1024 shots / half all <Z_i>", "requests": count, "gates": G,
                   "rates": rates, "hbm_budget_GB": budget / 1e9, "arena_GB": arena / 1e9, "lanes": args.lanes,
                   "seed": args.seed, "l2": "no flush: per-request states, most larger than L2 at the top sizes"},
        "p50_ms": top["p50_ms"], "p99_ms": top["p99_ms"], "sweep": sweep,
        "plain_per_circuit_path": {"circuits_per_s": plain_rate, "sample": len(sample),
                                   "service_p50_ms": float(np.percentile(svc, 50) * 1e3),
                                   "service_p99_ms": float(np.percentile(svc, 99) * 1e3),
                                   "what": "per-gate kernels + readout, one request at a time, no queueing "
                                           "(service time only: a lower bound on its latency)"},
        "speedup_vs_plain": top["circuits_per_s"] / plain_rate,
        "accuracy": {"max_one_minus_F": max_inf, "max_abs_dZ": max_dz, "sample_max_qubits": 26,
                     "tolerance": {"one_minus_F": 1e-5}},
        "results_identical_across_rates": same,
        "host_circuit_build_s": build_s,
        "e2e": {"value": top["circuits_per_s"], "unit": "circuits/s",
                "h2d_bytes_per_step": h2d_step, "d2h_bytes_per_step": d2h_step,
                "timing": "host wall clock from first submit to last result; each request's plan tables and "
                          "uniforms go host->device, its <Z_i> or outcomes device->host, inside the span"},
        "cpu_baseline": cpu, "gpu_launches": launches * len(rates), "clocks": clk,
    }
    for c in circs:
        c.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--qubits", type=int, default=30)
    ap.add_argument("--depth", type=int, default=40)
    ap.add_argument("--circuit", default="brickwork", choices=["brickwork", "qft"],
                    help="plain form circuit: random brickwork (headline) or the QFT")
    ap.add_argument("--dtype", default="c64", choices=["c64", "c128"])
    ap.add_argument("--mode", default="auto", choices=["auto", "tiled", "pergate", "fused", "tensor"],
                    help="engine mode of the plain form; auto = the engine's NQPU_MODE_AUTO choice")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--tile-ctas", type=int, default=0, help="tiled kernel CTAs per SM (1 or 2; 0 = library default)")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-budget-s", type=float, default=15.0)
    ap.add_argument("--ref-step-s", type=float, default=4.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--quick", action="store_true", help="timed region only (profiling runs)")
    ap.add_argument("--form", default="plain", choices=["plain", "precision", "batch", "serve"],
                    help="plain: 30q brickwork (headline); precision: 32q TFIM fused tensor-core form; "
                         "batch: 4096 mixed-size HEA circuits in one persistent launch; "
                         "serve: Poisson request streams through the request loop")
    ap.add_argument("--tfim-steps", type=int, default=100)
    ap.add_argument("--circuits", type=int, default=4096, help="batch form: circuits per batch")
    ap.add_argument("--tune-sample", type=int, default=1024, help="batch form: autotuner sample size")
    ap.add_argument("--plain-sample", type=int, default=64, help="batch form: plain-path sample size")
    ap.add_argument("--no-tune-cache", action="store_true")
    ap.add_argument("--requests", type=int, default=400, help="serve form: requests per offered rate")
    ap.add_argument("--rates", default="20,40,80,160,320,640",
                    help="serve form: offered rates (requests/s); the last one saturates the server")
    ap.add_argument("--lanes", type=int, default=16, help="serve form: concurrent requests on the device")
    ap.add_argument("--serve-budget-gb", type=float, default=64.0, help="serve form: HBM budget for states")
    ap.add_argument("--embedded-rates", default="40,160,640",
                    help="serve rates of the serve block inside the default (plain) line")
    ap.add_argument("--plain-only", action="store_true",
                    help="default run: only the plain 30q line (no config-1, precision, batch, serve blocks)")
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and not args.quick:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.form == "batch":
        print(json.dumps(run_batch(args)), flush=True)
    elif args.form == "serve":
        print(json.dumps(run_serve(args)), flush=True)
    elif args.form == "precision":
        if args.qubits == 30:
            args.qubits = 32
        print(json.dumps(run_precision(args)), flush=True)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
