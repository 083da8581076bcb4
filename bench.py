#!/usr/bin/env python
"""RGF transport benchmark: energy-point solves/s on one or more B200s.

Workload (the single-GPU scale-up): a seeded block-tridiagonal device with
nb = 64 blocks of b = 256 orbitals, 1024 energies on [-2, 2], complex128.
One step = one batch of energies (by default one energy per SM, 148 on a
B200: the block inverse runs one matrix per SM, so the batch fills exactly
one wave of it) through the full hot path:
A(E) = (E + i eta) I - H formed on the device, Sancho-Rubio for both contacts
(tol 1e-12), contact self-energies, the RGF selected solve returning the
diagonal and first off-diagonal blocks of G^R, G^< and G^>, per-block density,
contact currents and the Caroli transmission.  With the defaults
(--steps 7, 148 energies per step) the timed region covers all 1024 energies
(1036 solves; steps wrap around the energy grid).

value: whole-job solves/s with H resident in HBM; e2e: the same through the
public API with H and the energies copied from pinned host memory and the
step's observables (density, currents, transmission) read back every step.
Under torchrun each rank solves its own energies (weak scaling, no collective
on the data path); the time is the maximum over ranks.

--impl reference times the CPU implementation of the same path (the NumPy
restatement of the upstream algorithm in oracle/) on the host cores.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FP64_DMMA_PEAK_TFLOPS = 37.0  # measured on this pool's B200s: mma.sync m8n8k4 f64 issue-rate probe
FP64_PEAK_SOURCE = "measured: DMMA issue-rate probe on B200 (profiles/fp64_peak_b200.md)"
GEMM_TRAFFIC_BYTES = 373.1e6  # zgemm_dmma_kernel, b = 256, batch 128: 269.0 MB read + 104.1 MB written
OZAKI_TRAFFIC_BYTES = 459.7e6  # ozaki_gemm_kernel, same shape: 352.7 MB read (slices) + 107.0 MB written


def _workload(args):
    from quatrex_b200.workloads import CONFIG_LARGE, CONFIG_SMALL

    cfg = dict(CONFIG_LARGE if args.workload == "large" else CONFIG_SMALL)
    return cfg


def _flops_per_energy(nb, b, sr_iterations):
    """Algorithmic flops of one energy solve of the generator form (zero interior
    self-energies), in units of one b x b complex product (8 b^3 flops; a block
    inverse counts as one), as executed: the Keldysh recursion runs for the two
    contact sources (X_L from block 0, X_R from block nb - 1; X_R is zero in the
    forward sweep):
      first block: inverse + 2 products for X_L,0                   =  3
      forward step: A_ji x_i, Schur update, inverse,
                    3 for X_L (W = x_j A_ji, W X W^H)             =  6 per step
      last block: 2 products for X_R                                =  2
      backward step: P1, P2, P4, G^R_ij, G^R_ji, corner chain,
                     4 for X_L, 2 for X_R, x_i                      = 13 per step
      contacts: Sigma^R 2 x 2; transmission: 2                      =  6
      Sancho-Rubio: 7 per iteration + final inverse, per contact"""
    units = 3 + 2 + (nb - 1) * (6 + 13) + 6 + sum(7 * it + 1 for it in sr_iterations)
    return 8.0 * b ** 3 * units


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, local_index: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        ids = [v.strip() for v in vis.split(",")] if vis else []
        self.index = ids[local_index] if local_index < len(ids) else str(local_index)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(cfg, sample_energies: int, threads_note: dict):
    """The oracle (NumPy restatement of the upstream path) on a bounded sample."""
    from oracle import rgf_oracle as orc
    from quatrex_b200.workloads import make_device

    dev = make_device(**cfg)
    idx = np.linspace(0, cfg["num_energies"] - 1, sample_energies).round().astype(int)
    e = dev.energies[idx]
    results = []
    t0 = time.perf_counter()
    for k in range(len(e)):
        ek = e[k:k + 1]
        d, u, lo = dev.system_blocks(ek)
        obc = orc.obc_self_energies(d, u, lo, ek, dev.mu_left, dev.mu_right, dev.kt, dev.sr_tol, dev.sr_max_iter)
        nb = len(d)
        pad = [None] * (nb - 2)
        z = [np.zeros_like(x) for x in d]
        zu = [np.zeros_like(x) for x in u]
        ref = orc.selected_solve(d, u, lo, z, zu, z, zu, [obc["retarded"][0], *pad, obc["retarded"][1]],
                                 [obc["lesser"][0], *pad, obc["lesser"][1]],
                                 [obc["greater"][0], *pad, obc["greater"][1]], return_extras=True)
        trans = orc.caroli_transmission(ref["xr_corner"], obc["gamma"][0], obc["gamma"][1])
        dens = orc.block_density(ref["xl_diag"])
        results.append({"gr_diag": np.stack(ref["xr_diag"], axis=1)[0], "gl_diag": np.stack(ref["xl_diag"], axis=1)[0],
                        "density": dens[0], "transmission": float(trans[0])})
    dt = time.perf_counter() - t0
    return len(e) / dt, dt, idx, results


def accuracy_against_oracle(gpu: dict, oracle_results: list) -> dict:
    """Largest error over the sampled energies of one GPU form against the
    oracle (end to end: the oracle's own Sancho-Rubio): G^R and G^< diagonal
    blocks (relative Frobenius per block), per-block density (relative to the
    energy's largest block), transmission (relative)."""
    err = {"gr_diag_block_rel_max": 0.0, "gl_diag_block_rel_max": 0.0, "density_rel_max": 0.0,
           "transmission_rel_max": 0.0}
    for k, ref in enumerate(oracle_results):
        for key, name in (("gr_diag", "gr_diag_block_rel_max"), ("gl_diag", "gl_diag_block_rel_max")):
            got = gpu[key][k]
            num = np.linalg.norm(got - ref[key], axis=(-2, -1))
            den = np.maximum(np.linalg.norm(ref[key], axis=(-2, -1)), 1e-300)
            err[name] = max(err[name], float((num / den).max()))
        err["density_rel_max"] = max(err["density_rel_max"], float(
            np.abs(gpu["density"][k] - ref["density"]).max() / max(np.abs(ref["density"]).max(), 1e-300)))
        err["transmission_rel_max"] = max(err["transmission_rel_max"], float(
            abs(gpu["transmission"][k] - ref["transmission"]) / max(abs(ref["transmission"]), 1e-12)))
    return err


def blas_threads() -> dict:
    try:
        from threadpoolctl import threadpool_info

        info = threadpool_info()
        blas = [i for i in info if i.get("user_api") == "blas"]
        if blas:
            return {"threads": int(blas[0].get("num_threads", 1)), "library": blas[0].get("internal_api", "?")}
    except Exception:
        pass
    return {"threads": os.cpu_count() or 1, "library": "?"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    cfg = _workload(args)
    bt = blas_threads()
    total = 0.0
    solves = 0
    # warm-up: one energy each
    for _ in range(args.warmup):
        cpu_baseline(cfg, 1, bt)
    for _ in range(args.steps):
        rate, dt, _, _ = cpu_baseline(cfg, args.ref_energies_per_step, bt)
        total += dt
        solves += args.ref_energies_per_step
    value = solves / total
    sample = (f"{args.ref_energies_per_step} energy solve(s) per step of nb={cfg['num_blocks']}, "
              f"b={cfg['block_size']} (Sancho-Rubio both contacts + selected solve + transmission)")
    line = {
        "impl": "reference", "metric": "rgf_energy_solves_per_s", "value": value, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "complex128", "data": "synthetic (seeded generator)",
        "config": {"workload": f"transport nb={cfg['num_blocks']} b={cfg['block_size']} "
                               f"E={cfg['num_energies']} complex128", "energies_per_step": args.ref_energies_per_step},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": bt["threads"], "kind": "port",
                         "sample": sample, "blas": bt["library"]},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist

    from quatrex_b200 import _lib
    from quatrex_b200.energy_shards import max_over_ranks
    from quatrex_b200.transport import TransportSolver
    from quatrex_b200.workloads import make_device

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device(f"cuda:{local}"))

    def barrier():
        if world > 1:
            dist.barrier()

    cfg = _workload(args)
    dev = make_device(**cfg)
    E = args.energies_per_step
    if E <= 0:
        E = torch.cuda.get_device_properties(local).multi_processor_count
    nb, b = cfg["num_blocks"], cfg["block_size"]
    solver = TransportSolver(dev, max_batch_size=E, precision=args.precision, cuda_device=local)
    energies_all = torch.from_numpy(dev.energies).to(f"cuda:{local}")
    out = solver.allocate_outputs(E)
    n_all = len(dev.energies)

    def step_energies(k):
        g = (k * world + rank) * E
        idx = (torch.arange(E, device=f"cuda:{local}") + g) % n_all
        return energies_all[idx].contiguous()

    stream = torch.cuda.current_stream()
    step_e = [step_energies(k) for k in range(args.steps)]
    for k in range(args.warmup):
        solver.solve(step_energies(k), out)
    torch.cuda.synchronize()

    # ---- device-resident timed region
    ctx_launch0 = _lib.launch_count(local)
    _lib.set_timing(True, local)
    sr_its = []
    with ClockSampler(local) as clocks:
        barrier()
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for k in range(args.steps):
            solver.solve(step_e[k], out)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    elapsed_ms = ev0.elapsed_time(ev1)
    launches = _lib.launch_count(local) - ctx_launch0
    gemm = _lib.timing_report(0, local)
    inv = _lib.timing_report(1, local)
    _lib.set_timing(False, local)
    sr_its = out["sr_iterations"].cpu().numpy()
    elapsed_ms = max_over_ranks(elapsed_ms, device=f"cuda:{local}")
    value = world * args.steps * E / (elapsed_ms / 1000.0)

    # ---- end to end through the public API (TransportSolver.solve over
    # qtx_transport_solve): every step copies H and its energies in from
    # pinned host memory and copies back to pinned host memory every diagonal
    # block of G^R, G^< and G^> (the blocks the density, the DOS and the
    # carrier statistics are read from) plus the observables.  The outputs are
    # double buffered on the device so that the download of step k runs on a
    # copy stream while step k + 1 solves; the timed region ends when the
    # last download has landed.
    del out
    torch.cuda.empty_cache()
    e2e = None
    if not args.no_e2e:
        e2e = _e2e_generator(args, dev, E, step_energies, stream, barrier, local, world)

    # ---- roofline of the dominant kernel (batched complex FP64 GEMM on DMMA)
    gemm_tflops = gemm["flops"] / (gemm["ms"] / 1000.0) / 1e12 if gemm["ms"] > 0 else 0.0
    roofline = {
        "kernel": "zgemm_dmma_kernel", "bound": "tensor", "achieved": round(gemm_tflops, 3),
        "peak": FP64_DMMA_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": round(gemm_tflops / FP64_DMMA_PEAK_TFLOPS, 4),
        "peak_source": FP64_PEAK_SOURCE,
        # DRAM bytes of one launch of this kernel at the bench shape (b = 256, 128 energies), from one ncu
        # capture; the algorithmic minimum is 402.7 MB (A, B read, D written once)
        "traffic": GEMM_TRAFFIC_BYTES,
        "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/zgemm_dmma_b256_batch128.md",
        "gemm_launches": gemm["launches"], "gemm_ms": round(gemm["ms"], 3),
        "gemm_share_of_step": round(gemm["ms"] / elapsed_ms, 4) if elapsed_ms > 0 else None,
        "inverse_ms": round(inv["ms"], 3), "inverse_launches": inv["launches"],
        "inverse_tflops": round(inv["flops"] / (inv["ms"] / 1000.0) / 1e12, 3) if inv["ms"] > 0 else None,
        "inverse_frac": (round(inv["flops"] / (inv["ms"] / 1000.0) / 1e12 / FP64_DMMA_PEAK_TFLOPS, 4)
                         if inv["ms"] > 0 else None),
    }
    alg = _flops_per_energy(nb, b, [float(np.mean(sr_its[:, 0])), float(np.mean(sr_its[:, 1]))])
    whole_tflops = alg * args.steps * E / (elapsed_ms / 1000.0) / 1e12

    if args.precision == "mixed":
        roofline["kernel"] = ("complex GEMM class: ozaki_split + ozaki_gemm_kernel (INT8 tcgen05) in the sweep, "
                              "zgemm_dmma_kernel in Sancho-Rubio; FP64-equivalent flops")
        roofline["traffic"] = OZAKI_TRAFFIC_BYTES
        roofline["traffic_source"] = "ncu capture of ozaki_gemm_kernel, profiles/ozaki_gemm_b256_batch128.md"

    # ---- the precision form on the same workload, same box, same run (rank 0
    # alone, device resident): its rate and its ratio to this line's form
    mixed = None
    if args.precision == "fp64" and world == 1 and not args.no_mixed:
        mixed = _mixed_line(args, dev, E, step_energies, stream, local, value)

    # ---- CPU baseline (the oracle on a bounded sample) and the accuracy of
    # the FP64 and mixed forms against it at the same energies
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        bt = blas_threads()
        rate, dt, idx, oracle_results = cpu_baseline(cfg, args.cpu_energies, bt)
        cpu = {"value": rate, "unit": "solves/s", "cores": bt["threads"], "kind": "port",
               "sample": f"{args.cpu_energies} energies of the same workload ({dt:.1f} s, oracle NumPy path)",
               "blas": bt["library"]}
        e_chk = torch.from_numpy(dev.energies[idx]).to(f"cuda:{local}")
        keys = ("gr_diag", "gl_diag", "density", "transmission")
        acc = {}
        for prec in ("fp64", "mixed"):
            if prec == "mixed" and mixed is None:
                continue
            res = TransportSolver(dev, max_batch_size=len(idx), precision=prec, cuda_device=local).solve(
                e_chk, keys=keys)
            acc[prec] = accuracy_against_oracle({k: v.cpu().numpy() for k, v in res.items()}, oracle_results)
            del res
        cpu["accuracy_fp64"] = acc["fp64"]
        if mixed is not None:
            mixed["accuracy"] = acc["mixed"]
            mixed["accuracy"]["against"] = (f"oracle (NumPy, end to end incl. its Sancho-Rubio) at energy "
                                            f"indices {idx.tolist()}")

    if rank == 0:
        line = {
            "metric": "rgf_energy_solves_per_s", "value": round(value, 3), "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(elapsed_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "complex128",
            "data": "synthetic (seeded Hamiltonian generator)",
            "config": {
                "workload": f"transport nb={nb} b={b} E={cfg['num_energies']} complex128, "
                            f"{args.precision}", "energies_per_step": E, "precision": args.precision,
                "l2": "inputs larger than L2 (per-step state >= 24 GB)", "parallelism": f"energy shards x{world}"},
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "whole_step_tflops_fp64_equiv": round(whole_tflops, 3),
            "sr_iterations_mean": [float(np.mean(sr_its[:, 0])), float(np.mean(sr_its[:, 1]))],
        }
        if mixed is not None:
            line["mixed"] = mixed
        if world == 1 and not args.no_dropin_e2e:
            line["e2e_dropin"] = _e2e_dropin(args)
        if world == 1 and not args.no_serve:
            torch.cuda.empty_cache()
            line["serve"] = {ln["precision"]: {k: v for k, v in ln.items()
                                               if k not in ("metric", "impl", "workload", "precision")}
                             for ln in serve_lines(args)}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


E2E_KEYS = ("gr_diag", "gl_diag", "gg_diag", "density", "hole_density", "transmission", "current_left",
            "current_right", "dos", "sr_iterations")


def _e2e_generator(args, dev, E, step_energies, stream, barrier, local, world):
    import torch

    from quatrex_b200.energy_shards import max_over_ranks
    from quatrex_b200.transport import TransportSolver

    cuda = f"cuda:{local}"
    h_diag_host = torch.from_numpy(dev.h_diag).pin_memory()
    h_upper_host = torch.from_numpy(dev.h_upper).pin_memory()
    e_host = [step_energies(k).cpu().pin_memory() for k in range(args.steps)]
    h_diag_dev = torch.empty(h_diag_host.shape, dtype=h_diag_host.dtype, device=cuda)
    h_upper_dev = torch.empty(h_upper_host.shape, dtype=h_upper_host.dtype, device=cuda)
    e_dev = torch.empty(E, dtype=torch.float64, device=cuda)
    solver = TransportSolver(dev, max_batch_size=E, precision=args.precision, cuda_device=local,
                             h_diag=h_diag_dev, h_upper=h_upper_dev)
    bufs = [solver.allocate_outputs(E, keys=E2E_KEYS) for _ in range(2)]
    # one flat page-locked host buffer holds every returned array of a step
    sizes = {k: v.numel() * v.element_size() for k, v in bufs[0].items()}
    total = sum((n + 255) // 256 * 256 for n in sizes.values())
    flat = torch.empty(total, dtype=torch.uint8, pin_memory=True)
    host, off = {}, 0
    for k, v in bufs[0].items():
        host[k] = flat[off:off + sizes[k]].view(v.dtype).view(v.shape)
        off += (sizes[k] + 255) // 256 * 256
    copy_stream = torch.cuda.Stream(device=cuda)
    h2d = h_diag_host.numel() * 16 + h_upper_host.numel() * 16 + E * 8
    d2h = sum(sizes.values())

    def one_step(k, timed_events):
        kb = k % 2
        stream.wait_event(timed_events["copied"][kb])  # buffer kb's previous download has landed
        h_diag_dev.copy_(h_diag_host, non_blocking=True)
        h_upper_dev.copy_(h_upper_host, non_blocking=True)
        e_dev.copy_(e_host[k % len(e_host)], non_blocking=True)
        solver.solve(e_dev, bufs[kb])
        timed_events["solved"][kb].record(stream)
        copy_stream.wait_event(timed_events["solved"][kb])
        with torch.cuda.stream(copy_stream):
            for key, t in bufs[kb].items():
                host[key].copy_(t, non_blocking=True)
        timed_events["copied"][kb].record(copy_stream)

    ev = {"solved": [torch.cuda.Event() for _ in range(2)], "copied": [torch.cuda.Event() for _ in range(2)]}
    for e in ev["copied"]:
        e.record(copy_stream)
    for k in range(args.warmup):
        one_step(k, ev)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.steps):
        one_step(k, ev)
    stream.wait_stream(copy_stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(ev0.elapsed_time(ev1), device=cuda)
    # the host copy of the last step is the solve's result: spot-check it is there
    assert torch.isfinite(host["density"]).all()
    del bufs, flat, host
    torch.cuda.empty_cache()
    return {"value": world * args.steps * E / (e2e_ms / 1000.0), "unit": "solves/s",
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "ms_per_step": round(e2e_ms / args.steps, 3),
            "returned": "every diagonal block of G^R, G^<, G^> + density, hole density, DOS, transmission, "
                        "contact currents (double-buffered on the device, downloads overlap the next solve)",
            "path": "TransportSolver.solve -> qtx_transport_solve, H and energies from pinned host memory"}


def _mixed_line(args, dev, E, step_energies, stream, local, fp64_value):
    import torch

    from quatrex_b200.transport import TransportSolver

    solver = TransportSolver(dev, max_batch_size=E, precision="mixed", cuda_device=local)
    keys = ("gr_diag", "gr_upper", "gr_lower", "gl_diag", "gl_upper", "gg_diag", "gg_upper", "density",
            "hole_density", "transmission", "current_left", "current_right", "sr_iterations", "dos", "layer_current")
    out = solver.allocate_outputs(E, keys)
    step_e = [step_energies(k) for k in range(args.steps)]
    for k in range(args.warmup):
        solver.solve(step_energies(k), out)
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(args.steps):
        solver.solve(step_e[k], out)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    del out
    torch.cuda.empty_cache()
    v = args.steps * E / (ms / 1000.0)
    return {"value": round(v, 3), "unit": "solves/s", "ms_per_step": round(ms / args.steps, 3),
            "ratio_vs_fp64": round(v / fp64_value, 4), "steps": args.steps, "warmup": args.warmup,
            "form": "bulk sweep products as INT8 split products (tcgen05 kind::i8, 8 slices), inverses and "
                    "Sancho-Rubio in FP64; same outputs as the FP64 line"}


def _e2e_dropin(args):
    """The plugin call RGF.selected_solve(return_retarded) on NumPy DSDBCOO
    matrices of the nb=64, b=256 device (32 energies, batches of 16): every
    operand streamed host -> device and every output block back inside the
    timed region (QTX_FLAG_HOST_BUFFERS)."""
    import torch

    from quatrex_b200.datastructures import DSDBCOO
    from quatrex_b200.greens_function_solver import RGF, OBCBlocks
    from quatrex_b200.obc import SanchoRubio, contact_self_energies
    from quatrex_b200.workloads import make_device

    nb, b, ne, batch = 64, 256, 32, 16
    dev = make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=1234)
    d, u, lo = dev.system_blocks()
    A = DSDBCOO.from_blocks(d, u, lo)
    Z = DSDBCOO.zeros_like(A)
    e = dev.energies
    sr = SanchoRubio(dev.sr_max_iter, dev.sr_tol)
    g_left = sr(d[0], u[0], lo[0])
    g_right = sr(d[-1], lo[-1], u[-1])
    f_left = 1.0 / (1.0 + np.exp((e - dev.mu_left) / dev.kt))
    f_right = 1.0 / (1.0 + np.exp((e - dev.mu_right) / dev.kt))
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.lesser[0], ob.greater[0] = contact_self_energies(g_left, lo[0], u[0], f_left)
    ob.retarded[-1], ob.lesser[-1], ob.greater[-1] = contact_self_energies(g_right, u[-1], lo[-1], f_right)
    del d, u, lo
    outs = [DSDBCOO.zeros_like(A) for _ in range(3)]
    solver = RGF(max_batch_size=batch)
    for _ in range(2):
        solver.selected_solve(A, Z, Z, obc_blocks=ob, out=outs, return_retarded=True)
    torch.cuda.synchronize()
    steps = 2
    t0 = time.perf_counter()
    for _ in range(steps):
        solver.selected_solve(A, Z, Z, obc_blocks=ob, out=outs, return_retarded=True)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    row_bytes = A.data.shape[-1] * 16
    return {"value": round(ne * steps / dt, 3), "unit": "solves/s", "h2d_bytes_per_step": int(3 * ne * row_bytes),
            "d2h_bytes_per_step": int(3 * ne * row_bytes), "steps": steps, "warmup": 2,
            "path": "RGF.selected_solve(a, sigma_lesser, sigma_greater, obc_blocks, out=[xl, xg, xr], "
                    "return_retarded=True) on NumPy DSDBCOO -> qtx_selected_solve with QTX_FLAG_HOST_BUFFERS",
            "config": {"num_blocks": nb, "block_size": b, "energies": ne, "max_batch_size": batch,
                       "outputs": "G^<, G^> (every BTD block), G^R diagonal; Sigma^<, Sigma^> zero in the interior"}}


def run_uneven(args):
    """Uneven batch: a seeded prefix of instances drawn with the uneven-batch size
    distribution (b log-uniform over 32..512, nb uniform in [8, 128], 64-512
    energies), solved with concurrent streams, both precisions."""
    import torch

    from quatrex_b200.autotune import Autotuner
    from quatrex_b200.batching import BatchedTransport, Instance, total_flops, total_solves
    from quatrex_b200.workloads import make_device, uneven_instances

    draws = uneven_instances(args.instances, seed=4321)
    insts = [Instance(make_device(**d), None) for d in draws]
    for x in insts:
        x.energies = x.device.energies
    lines = []
    if args.uneven_precision == "both":
        # each precision in a fresh process: the device memory pools, graph
        # memory and autotuner probes of one run do not weigh on the other
        rc = 0
        for prec in ("fp64", "mixed"):
            cmd = [sys.executable, os.path.abspath(__file__), "--workload", "uneven", "--instances",
                   str(args.instances), "--streams", str(args.streams), "--uneven-precision", prec]
            if args.no_group:
                cmd.append("--no-group")
            rc = rc or subprocess.call(cmd)
        return rc
    for prec in (args.uneven_precision,):
        tuner = Autotuner(cache_path=os.path.join(ROOT, "_build", "autotune.json"))
        bt = BatchedTransport(precision=prec, streams=args.streams, tuner=tuner, group_small=not args.no_group)
        try:
            # warm-up outside the timed region: tune every (b, batch, precision)
            # key the instances use, then run the smallest instance once
            for kind, idx in bt.jobs(insts):
                if kind == "one":
                    bt.choice_for(insts[idx[0]])
            bt.run([min(insts, key=lambda x: x.device.block_size * x.device.num_blocks)])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = bt.run(insts)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            per_instance = [{"b": x.device.block_size, "nb": x.device.num_blocks, "ne": len(x.energies),
                             "seconds": round(r["seconds"], 3),
                             "choice": ({"path": "grouped persistent launch (fp64)"} if r["grouped"] else
                                        {k: v for k, v in bt.choice_for(x).items() if k != "probe_solves_per_s"})}
                            for x, r in zip(insts, res)]
        finally:
            bt.close()
        lines.append({"metric": "rgf_energy_solves_per_s", "impl": "ours", "workload": "uneven",
                      "precision": prec, "value": total_solves(insts) / dt, "unit": "solves/s",
                      "seconds": dt, "instances": len(insts), "solves": total_solves(insts),
                      "alg_tflops": total_flops(insts) / dt / 1e12, "streams": args.streams,
                      "grouped_small": not args.no_group,
                      "per_instance": per_instance})
        print(json.dumps(lines[-1]), flush=True)
    return 0


def run_serve(args):
    """Serving: a seeded Poisson stream of requests (b in 32..256, nb 8..32,
    16-64 energies each), continuous batching, both precisions; p50/p99."""
    for line in serve_lines(args):
        print(json.dumps(line), flush=True)
    return 0


def serve_lines(args) -> list:
    """The serving measurement of run_serve, one dict per precision."""
    import torch

    from quatrex_b200.autotune import Autotuner
    from quatrex_b200.serving import TransportServer, poisson_arrivals
    from quatrex_b200.workloads import make_device, uneven_instances

    reqs = []
    if getattr(args, "serve_sizes", "small") == "uneven":
        # the size distribution of the uneven-instance batch (b up to 512, nb up to 128, 64-512 energies)
        for k, kw in enumerate(uneven_instances(args.requests, seed=99)):
            reqs.append(make_device(**kw))
        drawn = "seeded: the uneven-batch distribution, b = 2^U{5..9}, nb U[8, 128], 64-512 energies"
    else:
        rng = np.random.default_rng(99)
        for k in range(args.requests):
            b = int(2 ** rng.integers(5, 9))
            nb = int(rng.integers(8, 33))
            ne = int(rng.integers(16, 65))
            reqs.append(make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=5000 + k))
        drawn = "seeded: b = 2^U{5..8}, nb U[8, 32], 16-64 energies"
    arrivals = poisson_arrivals(len(reqs), rate_hz=args.rate, seed=7)
    lines = []
    precs = ("fp64", "mixed") if getattr(args, "serve_precision", "both") == "both" else (args.serve_precision,)
    for prec in precs:
        tuner = Autotuner(cache_path=os.path.join(ROOT, "_build", "autotune.json"))
        server = TransportServer(slots=args.streams, precision=prec, tuner=tuner, group_small=not args.no_group)
        try:
            # warm-up outside the timed region: tune every (b, batch, precision)
            # key the requests use, and run one request of each block size alone
            for d in reqs:
                tuner.best(d.block_size, len(d.energies), prec)
            seen = set()
            for d in reqs:
                if d.block_size not in seen:
                    seen.add(d.block_size)
                    server.submit(d, d.energies[:8]).result()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            futs = []
            for d, t in zip(reqs, arrivals):
                while time.perf_counter() - t0 < t:
                    time.sleep(0.0002)
                futs.append(server.submit(d, d.energies))
            results = [f.result() for f in futs]
            dt = time.perf_counter() - t0
            st = server.stats()
        finally:
            server.close()
        # latencies of the timed requests only (the server's own statistics include the warm-up)
        lat = np.array([r["latency_s"] for r in results])
        solves = int(sum(len(d.energies) for d in reqs))
        lines.append({"metric": "rgf_energy_solves_per_s", "impl": "ours", "workload": "serve",
                      "precision": prec, "value": solves / dt, "unit": "solves/s", "seconds": dt,
                      "requests": len(results), "p50_latency_s": float(np.percentile(lat, 50)),
                      "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
                      "peak_concurrency": st["peak_concurrency"], "arrival_rate_hz": args.rate,
                      "slots": args.streams, "server": "native qtx_server (C++ workers, one stream each)",
                      "grouped_small": not args.no_group,
                      "grouped_launches": st["grouped_launches"], "grouped_requests": st["grouped_requests"],
                      "requests_drawn": drawn})
    return lines


def run_dropin(args):
    """Drop-in plugin path: RGF.selected_solve (return_retarded) on DSDBCOO
    matrices of the seeded device, once with NumPy (host) data -- streamed
    through the device by QTX_FLAG_HOST_BUFFERS, host<->device copies inside
    the timed region -- and once with device-resident data."""
    import torch

    from quatrex_b200.datastructures import DSDBCOO
    from quatrex_b200.greens_function_solver import RGF, OBCBlocks
    from quatrex_b200.obc import SanchoRubio, contact_self_energies
    from quatrex_b200.workloads import make_device

    nb, b, ne = args.dropin_blocks, args.dropin_block_size, args.dropin_energies
    dev = make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=1234)
    d, u, lo = dev.system_blocks()
    A = DSDBCOO.from_blocks(d, u, lo)
    Z = DSDBCOO.zeros_like(A)
    e = dev.energies
    sr = SanchoRubio(dev.sr_max_iter, dev.sr_tol)
    g_left = sr(d[0], u[0], lo[0])
    g_right = sr(d[-1], lo[-1], u[-1])
    f_left = 1.0 / (1.0 + np.exp((e - dev.mu_left) / dev.kt))
    f_right = 1.0 / (1.0 + np.exp((e - dev.mu_right) / dev.kt))
    sig_l = contact_self_energies(g_left, lo[0], u[0], f_left)
    sig_r = contact_self_energies(g_right, u[-1], lo[-1], f_right)
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.lesser[0], ob.greater[0] = sig_l
    ob.retarded[-1], ob.lesser[-1], ob.greater[-1] = sig_r
    solver = RGF(max_batch_size=args.dropin_batch)
    lines = {}
    for where in ("host", "device"):
        if where == "host":
            a_, z_, obc = A, Z, ob
        else:
            a_, z_ = A.to("cuda"), Z.to("cuda")
            obc = OBCBlocks(nb)
            for lst_in, lst_out in ((ob.retarded, obc.retarded), (ob.lesser, obc.lesser), (ob.greater, obc.greater)):
                for i, x in enumerate(lst_in):
                    lst_out[i] = None if x is None else torch.from_numpy(x).cuda()
        outs = [DSDBCOO.zeros_like(a_) for _ in range(3)]
        for _ in range(args.warmup):
            solver.selected_solve(a_, z_, z_, obc_blocks=obc, out=outs, return_retarded=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            solver.selected_solve(a_, z_, z_, obc_blocks=obc, out=outs, return_retarded=True)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        lines[where] = ne * args.steps / dt
    row_bytes = A.data.shape[-1] * 16
    print(json.dumps({
        "metric": "rgf_energy_solves_per_s", "impl": "ours", "workload": "dropin_selected_solve",
        "value": lines["device"], "unit": "solves/s",
        "e2e": {"value": lines["host"], "unit": "solves/s", "h2d_bytes_per_step": int(6 * ne * row_bytes),
                "d2h_bytes_per_step": int(3 * ne * row_bytes),
                "path": "NumPy DSDBCOO -> QTX_FLAG_HOST_BUFFERS (streamed batches)"},
        "config": {"num_blocks": nb, "block_size": b, "energies": ne, "max_batch_size": args.dropin_batch,
                   "outputs": "G^<, G^> (all BTD blocks), G^R diagonal", "steps": args.steps},
    }), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=7)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["large", "small", "uneven", "serve", "dropin"], default="large")
    ap.add_argument("--dropin-blocks", type=int, default=16)
    ap.add_argument("--dropin-block-size", type=int, default=64)
    ap.add_argument("--dropin-energies", type=int, default=32)
    ap.add_argument("--dropin-batch", type=int, default=32)
    ap.add_argument("--instances", type=int, default=8, help="uneven workload: number of instances")
    ap.add_argument("--streams", type=int, default=4, help="uneven/serve: concurrent streams (slots)")
    ap.add_argument("--requests", type=int, default=48, help="serve workload: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="serve workload: Poisson arrival rate (1/s)")
    ap.add_argument("--serve-sizes", choices=["small", "uneven"], default="small",
                    help="serve workload: request sizes (small: b <= 256, nb <= 32; uneven: the uneven-batch draw)")
    ap.add_argument("--serve-precision", choices=["both", "fp64", "mixed"], default="both")
    ap.add_argument("--uneven-precision", choices=["both", "fp64", "mixed"], default="both")
    ap.add_argument("--no-group", action="store_true",
                    help="uneven/serve: solve b <= 64 instances (requests) one by one instead of grouped launches")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--energies-per-step", type=int, default=0,
                    help="energies per step (0: one per SM of the device)")
    ap.add_argument("--cpu-energies", type=int, default=3)
    ap.add_argument("--ref-energies-per-step", type=int, default=1)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the precision-form sub-line")
    ap.add_argument("--no-dropin-e2e", action="store_true", help="skip the plugin-call end-to-end key")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving (p50/p99) key")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "uneven":
        return run_uneven(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "dropin":
        return run_dropin(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
