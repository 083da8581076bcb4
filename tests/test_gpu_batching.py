"""Batching and serving forms on the GPU: CUDA-graph replay of the sweep,
uneven instances on concurrent streams, the continuous-batching server, and
the autotuner.  Every result must equal the same instance solved alone
(1e-12 relative; the kernels and batch composition of a request do not
depend on what else runs)."""

import json
import os
import time

import numpy as np
import pytest
import torch

from quatrex_b200 import _lib
from quatrex_b200.autotune import Autotuner
from quatrex_b200.batching import BatchedTransport, Instance, OBSERVABLE_KEYS
from quatrex_b200.serving import TransportServer, poisson_arrivals
from quatrex_b200.transport import TransportSolver, solve_grouped
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu


def _alone(dev, energies, ne_call, precision="fp64"):
    s = TransportSolver(dev, max_batch_size=ne_call, precision=precision)
    parts = []
    for c0 in range(0, len(energies), ne_call):
        parts.append(s.solve(energies[c0:c0 + ne_call], keys=OBSERVABLE_KEYS))
    return {k: torch.cat([p[k] for p in parts]).cpu().numpy() for k in OBSERVABLE_KEYS}


def _close(a, b, tol=1e-12):
    for k in ("density", "hole_density", "transmission", "current_left"):
        x, y = np.asarray(a[k]), np.asarray(b[k])
        assert np.linalg.norm(x - y) <= tol * max(np.linalg.norm(y), 1e-300), k


def test_graph_replay_matches_eager():
    dev = make_device(num_blocks=6, block_size=32, num_energies=8, seed=3)
    eager = TransportSolver(dev, max_batch_size=8).solve(dev.energies, keys=OBSERVABLE_KEYS)
    s = TransportSolver(dev, max_batch_size=8, use_graph=True)
    out = s.allocate_outputs(8, OBSERVABLE_KEYS)
    lib = _lib.load()
    ctx = _lib.context(torch.cuda.current_device())
    r0 = lib.qtx_graph_replays(ctx)
    for shift in (0.0, 0.01, 0.0):
        res = s.solve(dev.energies + shift, out)
        if shift == 0.0:
            for k in ("density", "transmission", "current_left"):
                assert torch.equal(res[k], eager[k]), k
    assert lib.qtx_graph_replays(ctx) - r0 == 3


@pytest.mark.parametrize("group", [False, True])
def test_uneven_instances_concurrent_streams(group):
    """With grouping, the b <= 64 instances of each block size share one
    persistent launch and equal the grouped solve of the instance alone bit for
    bit (a CTA's energy does not depend on the other pairs of the launch);
    larger instances, and every instance without grouping, equal the layered
    solve alone."""
    tuner = Autotuner(candidates_ne=(8,), repeats=1)
    insts = [Instance(make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=10 + i), None)
             for i, (nb, b, ne) in enumerate([(4, 16, 12), (7, 32, 9), (5, 64, 8), (3, 48, 17), (9, 16, 20),
                                              (3, 128, 6), (6, 64, 5)])]
    for x in insts:
        x.energies = x.device.energies
    bt = BatchedTransport(precision="fp64", streams=3, tuner=tuner, group_small=group)
    try:
        res = bt.run(insts)
    finally:
        bt.close()
    for x, r in zip(insts, res):
        assert r["grouped"] == (group and x.device.block_size <= 64)
        if r["grouped"]:
            alone = solve_grouped([x.device], [x.energies], keys=OBSERVABLE_KEYS)[0]
            for k in OBSERVABLE_KEYS:
                assert np.array_equal(r[k], alone[k].cpu().numpy()), k
        else:
            ne_call = tuner.best(x.device.block_size, len(x.energies), "fp64")["energies_per_call"]
            _close(r, _alone(x.device, x.energies, ne_call))


@pytest.mark.parametrize("group", [False, True])
def test_server_results_same_alone_and_in_mix(group):
    tuner = Autotuner(candidates_ne=(8,), repeats=1)
    rng = np.random.default_rng(1)
    devs = [make_device(num_blocks=int(rng.integers(3, 8)), block_size=int(rng.choice([16, 32, 64])),
                        num_energies=int(rng.integers(5, 20)), seed=100 + i) for i in range(8)]
    server = TransportServer(slots=3, precision="fp64", tuner=tuner, group_small=group)
    try:
        arrivals = poisson_arrivals(len(devs), rate_hz=200.0, seed=2)
        t0 = time.perf_counter()
        futs = []
        for d, t in zip(devs, arrivals):
            while time.perf_counter() - t0 < t:
                time.sleep(0.0005)
            futs.append(server.submit(d, d.energies))
        results = [f.result(timeout=300) for f in futs]
        st = server.stats()
    finally:
        server.close()
    assert st["completed"] == len(devs)
    assert st["p99_s"] >= st["p50_s"] > 0
    assert (st["grouped_requests"] == len(devs)) == group and st["grouped_launches"] <= st["grouped_requests"]
    for d, r in zip(devs, results):
        if group:
            # a grouped launch computes each energy on its own: the mix changes nothing
            alone = solve_grouped([d], [d.energies], keys=OBSERVABLE_KEYS)[0]
            for k in OBSERVABLE_KEYS:
                assert np.array_equal(r[k], alone[k].cpu().numpy()), k
        else:
            ne_call = tuner.best(d.block_size, len(d.energies), "fp64")["energies_per_call"]
            _close(r, _alone(d, d.energies, ne_call))


def test_server_rejects_request_above_budget():
    server = TransportServer(slots=1, memory_budget=1 << 20, tuner=Autotuner(candidates_ne=(8,), repeats=1))
    try:
        dev = make_device(num_blocks=8, block_size=64, num_energies=8, seed=1)
        with pytest.raises(MemoryError):
            server.submit(dev, dev.energies).result(timeout=60)
    finally:
        server.close()


def test_autotuner_persists(tmp_path):
    path = str(tmp_path / "tune.json")
    t = Autotuner(cache_path=path, candidates_ne=(8, 16), repeats=1)
    c = t.tune(32, 16, "mixed")
    assert c["energies_per_call"] in (8, 16) and c["gemm_path"] in ("fp64", "mixed")
    assert os.path.exists(path)
    t2 = Autotuner(cache_path=path)
    assert t2.lookup(32, 16, "mixed") == json.load(open(path))[Autotuner.key(32, 16, "mixed")]


def test_graph_scalars_in_key_and_release():
    """A captured sweep is replayed only for the scalars it was captured with,
    and released graphs are captured again on the next call."""
    import dataclasses

    dev = make_device(num_blocks=5, block_size=32, num_energies=6, seed=4)
    s = TransportSolver(dev, max_batch_size=6, use_graph=True)
    out = s.allocate_outputs(6, OBSERVABLE_KEYS)
    s.solve(dev.energies, out)
    dev2 = dataclasses.replace(dev, eta=1e-4, mu_left=dev.mu_left + 0.05)
    s2 = TransportSolver(dev2, max_batch_size=6, use_graph=True, h_diag=s.h_diag, h_upper=s.h_upper)
    s2._e_buf = s._e_buf  # same energy buffer: only the scalars differ from the first capture
    got = s2.solve(dev.energies, out)
    want = TransportSolver(dev2, max_batch_size=6).solve(dev.energies, keys=OBSERVABLE_KEYS)
    for k in ("density", "transmission", "current_left"):
        assert torch.equal(got[k], want[k]), k
    s.release_graphs()
    again = s.solve(dev.energies, out)
    ref = TransportSolver(dev, max_batch_size=6).solve(dev.energies, keys=OBSERVABLE_KEYS)
    for k in ("density", "transmission", "current_left"):
        assert torch.equal(again[k], ref[k]), k
