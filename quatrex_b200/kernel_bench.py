"""Fixed-shape launches of the hot kernels, timed with CUDA events.

``python -m quatrex_b200.kernel_bench gemm --b 256 --batch 128 --launches 5``
runs the batched complex GEMM of one RGF block product (b x b x b, ``batch``
energies) ``launches`` times after one warm-up launch and prints the mean
device time and TFLOP/s (8 b^3 flops per complex product).  ``inv`` does the
same for the batched block inverse (8 b^3 flops per block), ``sr`` for one
Sancho-Rubio solve.  ``grouped --b 32 --instances 6`` times the grouped
transport solve (one persistent launch for every energy of several seeded
devices of one block size, nb uniform in [8, 128], 64-512 energies; with
``--instances 1`` the single device nb=22 / 467 energies or, at b = 32,
nb=12 / 456 energies) against the layered solve of the same devices one after
the other, each after one warm-up call, with device-resident inputs.
``rgfdist --b 256 --nb 64 --energies 4 --partitions 2,4,8`` times the
selected solve of one seeded device by RGF and by RGFDist (partitions on
their own CUDA streams).  The same invocations are the targets of the ncu captures
summarised under profiles/.  Inputs are seeded, in HBM, and larger than L2 for
the default shapes (3 x 128 MiB operands at b = 256).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import sys

import numpy as np
import torch

from quatrex_b200 import _lib


def _rand(g, *shape):
    return torch.complex(torch.randn(*shape, generator=g, dtype=torch.float64),
                         torch.randn(*shape, generator=g, dtype=torch.float64)).cuda()


def bench_gemm(b: int, batch: int, launches: int, op_b: int = 0, precision: int = 0) -> dict:
    g = torch.Generator().manual_seed(1)
    a = _rand(g, batch, b, b)
    bb = _rand(g, batch, b, b)
    d = torch.empty_like(a)
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    s = torch.cuda.current_stream().cuda_stream

    def run():
        st = lib.qtx_zgemm(ctx, b, b, b, batch, 1.0, 0.0, a.data_ptr(), b, b * b, 0, bb.data_ptr(), b, b * b, op_b,
                           0.0, 0.0, None, b, b * b, d.data_ptr(), b, b * b, precision, s)
        _lib.check(st, ctx, "zgemm")

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(launches):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / launches
    flops = 8.0 * b ** 3 * batch
    ref = a[:2] @ (bb[:2] if op_b == 0 else bb[:2].conj().transpose(-1, -2))
    err = float(torch.linalg.norm(d[:2] - ref) / torch.linalg.norm(ref))
    return {"kernel": "zgemm", "b": b, "batch": batch, "ms": ms, "tflops": flops / ms / 1e9, "rel_err": err,
            "bytes_min": 3 * batch * b * b * 16}


def bench_inv(b: int, batch: int, launches: int) -> dict:
    rng = np.random.default_rng(2)
    a = rng.standard_normal((batch, b, b)) + 1j * rng.standard_normal((batch, b, b)) + np.sqrt(b) * np.eye(b)
    ta = torch.from_numpy(a).cuda()
    x = torch.empty_like(ta)
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    s = torch.cuda.current_stream().cuda_stream

    def run():
        _lib.check(lib.qtx_inv(ctx, b, batch, ta.data_ptr(), b * b, x.data_ptr(), b * b, s), ctx, "inv")

    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(launches):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / launches
    err = float(np.linalg.norm(x[:2].cpu().numpy() @ a[:2] - np.eye(b)) / np.sqrt(2 * b))
    return {"kernel": "zinv", "b": b, "batch": batch, "ms": ms, "tflops": 8.0 * b ** 3 * batch / ms / 1e9,
            "residual": err}


def bench_sr(b: int, batch: int, launches: int) -> dict:
    from quatrex_b200.obc import SanchoRubio
    from quatrex_b200.workloads import make_device

    dev = make_device(num_blocks=2, block_size=b, num_energies=batch, seed=5)
    d, u, lo = dev.system_blocks()
    tii = torch.from_numpy(d[0]).cuda()
    tij = torch.from_numpy(u[0][0]).cuda()
    tji = torch.from_numpy(lo[0][0]).cuda()
    sr = SanchoRubio(200, 1e-12)
    sr(tii, tij, tji)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(launches):
        sr(tii, tij, tji)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / launches
    it = float(np.mean(sr.last_iterations))
    return {"kernel": "sancho_rubio", "b": b, "batch": batch, "ms": ms, "mean_iterations": it,
            "tflops": 8.0 * b ** 3 * batch * (7 * it + 1) / ms / 1e9}


def bench_grouped(b: int, instances: int) -> dict:
    import time

    from quatrex_b200.batching import OBSERVABLE_KEYS
    from quatrex_b200.transport import TransportSolver, solve_grouped
    from quatrex_b200.workloads import make_device

    if instances == 1:
        specs = [(22, 467)] if b > 32 else [(12, 456)]
    else:
        rng = np.random.default_rng(0 if b == 32 else 1)
        specs = [(int(rng.integers(8, 129)), int(rng.integers(64, 513))) for _ in range(instances)]
    devs = [make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=900 + q) for q, (nb, ne) in enumerate(specs)]
    hs = [(torch.from_numpy(d.h_diag).cuda(), torch.from_numpy(d.h_upper).cuda()) for d in devs]
    es = [torch.from_numpy(d.energies).cuda() for d in devs]
    solves = sum(ne for _, ne in specs)

    def grouped():
        return solve_grouped(devs, es, keys=OBSERVABLE_KEYS, hamiltonians=hs)

    sols = [TransportSolver(d, max_batch_size=256, h_diag=h[0], h_upper=h[1]) for d, h in zip(devs, hs)]

    def layered():
        return [s.solve(e, keys=OBSERVABLE_KEYS) for s, e in zip(sols, es)]

    out = {}
    for name, fn in (("grouped", grouped), ("layered", layered)):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        out[name] = time.perf_counter() - t0
    return {"kernel": "transport_grouped", "b": b, "instances": [list(x) for x in specs], "solves": solves,
            "grouped_s": out["grouped"], "layered_s": out["layered"],
            "grouped_solves_per_s": solves / out["grouped"], "layered_solves_per_s": solves / out["layered"]}


def probe_fp64_peak() -> dict:
    from quatrex_b200.build import PROBE_LIB

    lib = ctypes.CDLL(PROBE_LIB)
    lib.qtx_probe_fp64_peak.restype = ctypes.c_int32
    lib.qtx_probe_fp64_peak.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
    out = {}
    for kind, name in ((0, "dmma_m8n8k4_tflops"), (1, "dfma_tflops")):
        v = ctypes.c_double()
        torch.cuda.init()
        st = lib.qtx_probe_fp64_peak(kind, ctypes.byref(v))
        if st != 0:
            raise RuntimeError(f"qtx_probe_fp64_peak failed with status {st}")
        out[name] = v.value
    return {"kernel": "fp64_peak_probe", **out}


def bench_rgfdist(b: int, nb: int, energies: int, partitions: list[int], repeats: int = 2) -> dict:
    """Selected solve of one seeded transport device (device-resident
    DSDBCOO operands, contact blocks, zero interior self-energies) by RGF and
    by RGFDist with each partition count; wall time per call after a
    warm-up call, and the largest per-block difference of G^< against RGF."""
    import time

    from quatrex_b200.datastructures import DSDBCOO
    from quatrex_b200.greens_function_solver import RGF, OBCBlocks
    from quatrex_b200.obc import SanchoRubio, contact_self_energies
    from quatrex_b200.rgf_dist import RGFDist
    from quatrex_b200.workloads import make_device

    dev = make_device(num_blocks=nb, block_size=b, num_energies=energies, seed=3)
    d, u, lo = dev.system_blocks()
    e = dev.energies
    sr = SanchoRubio(dev.sr_max_iter, dev.sr_tol)
    f_l = 1.0 / (1.0 + np.exp((e - dev.mu_left) / dev.kt))
    f_r = 1.0 / (1.0 + np.exp((e - dev.mu_right) / dev.kt))
    left = contact_self_energies(sr(d[0], u[0], lo[0]), lo[0], u[0], f_l)
    right = contact_self_energies(sr(d[-1], lo[-1], u[-1]), u[-1], lo[-1], f_r)
    A = DSDBCOO.from_blocks(d, u, lo, device="cuda")
    Z = DSDBCOO.zeros_like(A)
    ob = OBCBlocks(nb)
    ob.retarded[0], ob.lesser[0], ob.greater[0] = (torch.from_numpy(x).cuda() for x in left)
    ob.retarded[-1], ob.lesser[-1], ob.greater[-1] = (torch.from_numpy(x).cuda() for x in right)
    outs = [DSDBCOO.zeros_like(A) for _ in range(3)]

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(repeats):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / repeats

    rgf = RGF(max_batch_size=energies)
    t_rgf = timed(lambda: rgf.selected_solve(A, Z, Z, obc_blocks=ob, out=outs, return_retarded=True))
    ref = outs[0].data.clone()
    res = {"kernel": "rgf_vs_rgfdist", "b": b, "nb": nb, "energies": energies, "rgf_s": t_rgf}
    for p in partitions:
        solver = RGFDist(max_batch_size=energies, num_partitions=p)
        t = timed(lambda: solver.selected_solve(A, Z, Z, outs, ob, return_retarded=True))
        diff = float((outs[0].data - ref).abs().max() / ref.abs().max())
        res[f"rgfdist_p{p}_s"] = t
        res[f"rgfdist_p{p}_speedup"] = t_rgf / t
        res[f"rgfdist_p{p}_max_rel_diff_gl"] = diff
    return res


def bench_spectral(b: int, energies: int, rank: int, launches: int) -> dict:
    """Spectral OBC (Beyn contour NEVP + mode filter + surface recursion) and
    Sancho-Rubio on the same lead (cells coupled through ``rank`` boundary
    orbitals, make_lead), device-resident inputs: wall time per call after a
    warm-up call, and how far the two surface Green's functions agree."""
    import time

    from quatrex_b200.nevp import Beyn
    from quatrex_b200.obc import SanchoRubio, Spectral
    from quatrex_b200.workloads import make_lead

    a_ii, a_ij, a_ji, _ = make_lead(b, rank, energies, seed=11)
    dev = torch.cuda.current_device()
    tii = torch.from_numpy(a_ii).cuda(dev)
    tij = torch.from_numpy(np.ascontiguousarray(a_ij)).cuda(dev)
    tji = torch.from_numpy(np.ascontiguousarray(a_ji)).cuda(dev)
    m_0 = 4 * rank
    spec = Spectral(Beyn(r_o=10.0, r_i=0.8, m_0=m_0, num_quad_points=20))
    sr = SanchoRubio(max_iterations=200, convergence_tol=1e-12)

    def timed(fn):
        out = fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(launches):
            out = fn()
        torch.cuda.synchronize()
        return out, (time.perf_counter() - t0) / launches

    xs, t_spec = timed(lambda: spec(tii, tij, tji, "left"))
    xr, t_sr = timed(lambda: sr(tii, tij, tji, "left"))
    diff = torch.linalg.norm(xs - xr, dim=(-2, -1)) / torch.linalg.norm(xr, dim=(-2, -1))
    return {"kernel": "spectral_vs_sancho_rubio", "b": b, "energies": energies, "coupling_rank": rank, "m_0": m_0,
            "spectral_s": t_spec, "spectral_solves_per_s": energies / t_spec, "sancho_rubio_s": t_sr,
            "sancho_rubio_solves_per_s": energies / t_sr, "median_rel_diff": float(diff.median()),
            "sr_iterations_mean": float(np.mean(sr.last_iterations))}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="fixed-shape kernel timing")
    ap.add_argument("kernel", choices=["gemm", "gemm_h", "inv", "sr", "fp64peak", "grouped", "rgfdist", "spectral"])
    ap.add_argument("--rank", type=int, default=16, help="spectral: coupling rank of the lead")
    ap.add_argument("--nb", type=int, default=64)
    ap.add_argument("--energies", type=int, default=4)
    ap.add_argument("--partitions", type=str, default="2,4,8")
    ap.add_argument("--instances", type=int, default=6)
    ap.add_argument("--b", type=int, default=256)
    ap.add_argument("--batch", type=int, default=128)
    ap.add_argument("--launches", type=int, default=5)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    args = ap.parse_args(argv)
    prec = 0 if args.precision == "fp64" else 1
    if args.kernel == "fp64peak":
        r = probe_fp64_peak()
    elif args.kernel == "gemm":
        r = bench_gemm(args.b, args.batch, args.launches, 0, prec)
    elif args.kernel == "gemm_h":
        r = bench_gemm(args.b, args.batch, args.launches, 1, prec)
    elif args.kernel == "inv":
        r = bench_inv(args.b, args.batch, args.launches)
    elif args.kernel == "grouped":
        r = bench_grouped(args.b, args.instances)
    elif args.kernel == "spectral":
        r = bench_spectral(args.b, args.energies, args.rank, args.launches)
    elif args.kernel == "rgfdist":
        r = bench_rgfdist(args.b, args.nb, args.energies, [int(x) for x in args.partitions.split(",")])
    else:
        r = bench_sr(args.b, args.batch, args.launches)
    print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
