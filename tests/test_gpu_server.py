"""The native continuous-batching server (qtx_server_*) through the C ABI:
results equal a direct qtx_transport_solve of the same request, requests are
collected by id or in completion order, statistics add up, and requests over
the budget or malformed are refused at submission."""

import contextlib
import ctypes

import pytest
import torch

from quatrex_b200 import _lib
from quatrex_b200.transport import TransportSolver, allocate_outputs, solve_grouped
from quatrex_b200.workloads import make_device

pytestmark = pytest.mark.gpu
_nullcontext = contextlib.nullcontext

KEYS = ("density", "transmission", "current_left", "sr_iterations")


def _problem(dev, h_diag, h_upper, e, ne_call):
    return _lib.TransportProblem(
        num_blocks=dev.num_blocks, block_size=dev.block_size, num_energies=int(e.shape[0]),
        h_diag=h_diag.data_ptr(), h_upper=h_upper.data_ptr(), energies=e.data_ptr(), eta=dev.eta,
        mu_left=dev.mu_left, mu_right=dev.mu_right, kt=dev.kt, sr_tol=dev.sr_tol,
        sr_max_iterations=dev.sr_max_iter, max_batch_size=ne_call)


def _outputs(out):
    return _lib.TransportOutputs(**{name: (out[name].data_ptr() if name in out else None)
                                    for name, _ in _lib.TransportOutputs._fields_})


def _server(slots=3, budget=0, group=0):
    lib = _lib.load()
    cfg = _lib.ServerConfig(device=torch.cuda.current_device(), slots=slots, memory_budget=budget,
                            group_max_block_size=group)
    h = ctypes.c_void_p()
    assert lib.qtx_server_create(ctypes.byref(cfg), ctypes.byref(h)) == _lib.QTX_OK
    return lib, h.value


def test_native_server_matches_direct_solve():
    lib, srv = _server()
    devs = [make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=30 + i)
            for i, (nb, b, ne) in enumerate([(5, 32, 9), (7, 16, 12), (4, 64, 6), (6, 32, 10)])]
    keep, ids = [], []
    try:
        for d in devs:
            h_diag = torch.from_numpy(d.h_diag).cuda()
            h_upper = torch.from_numpy(d.h_upper).cuda()
            e = torch.from_numpy(d.energies).cuda()
            out = allocate_outputs(d.num_blocks, d.block_size, len(d.energies), KEYS, torch.cuda.current_device())
            torch.cuda.synchronize()
            p, o = _problem(d, h_diag, h_upper, e, 4), _outputs(out)
            rid = ctypes.c_int64()
            assert lib.qtx_server_submit(srv, ctypes.byref(p), ctypes.byref(o), _lib.QTX_PREC_FP64, 0,
                                         ctypes.byref(rid)) == _lib.QTX_OK
            keep.append((d, out, h_diag, h_upper, e, p, o))
            ids.append(rid.value)
        status, lat = ctypes.c_int32(), ctypes.c_double()
        # the last one by id, the others in completion order
        assert lib.qtx_server_wait(srv, ids[-1], -1, ctypes.byref(status), ctypes.byref(lat), None, 0) == 0
        assert status.value == _lib.QTX_OK and lat.value > 0
        got = {ids[-1]}
        rid = ctypes.c_int64()
        while len(got) < len(ids):
            st = lib.qtx_server_wait_any(srv, 60000, ctypes.byref(rid), ctypes.byref(status), ctypes.byref(lat),
                                         None, 0)
            assert st == _lib.QTX_OK and status.value == _lib.QTX_OK
            got.add(rid.value)
        assert got == set(ids)
        # collected ids are unknown afterwards
        assert lib.qtx_server_wait(srv, ids[0], 0, ctypes.byref(status), ctypes.byref(lat), None, 0) == \
            _lib.QTX_E_INVAL
        stats = _lib.ServerStats()
        assert lib.qtx_server_get_stats(srv, ctypes.byref(stats)) == 0
        assert stats.submitted == stats.completed == len(devs) and stats.failed == 0
        assert stats.solves == sum(len(d.energies) for d in devs)
        assert stats.p99_latency_s >= stats.p50_latency_s > 0 and stats.running == 0 and stats.queued == 0
    finally:
        assert lib.qtx_server_destroy(srv) == 0
    for d, out, *_ in keep:
        ref = TransportSolver(d, max_batch_size=4).solve(d.energies, keys=KEYS)
        for k in KEYS:
            assert torch.equal(out[k], ref[k]), k


def test_native_server_refuses_over_budget_and_bad_requests():
    lib, srv = _server(slots=1, budget=1 << 20)
    try:
        d = make_device(num_blocks=6, block_size=64, num_energies=8, seed=3)
        h_diag = torch.from_numpy(d.h_diag).cuda()
        h_upper = torch.from_numpy(d.h_upper).cuda()
        e = torch.from_numpy(d.energies).cuda()
        out = allocate_outputs(6, 64, 8, KEYS, torch.cuda.current_device())
        p, o = _problem(d, h_diag, h_upper, e, 8), _outputs(out)
        rid = ctypes.c_int64()
        need = lib.qtx_transport_footprint(6, 64, 8, _lib.QTX_PREC_FP64)
        assert need > (1 << 20)
        assert lib.qtx_server_submit(srv, ctypes.byref(p), ctypes.byref(o), 0, 0, ctypes.byref(rid)) == \
            _lib.QTX_E_NOMEM
        p.num_blocks = 1
        assert lib.qtx_server_submit(srv, ctypes.byref(p), ctypes.byref(o), 0, 0, ctypes.byref(rid)) == \
            _lib.QTX_E_INVAL
        status, lat = ctypes.c_int32(), ctypes.c_double()
        assert lib.qtx_server_wait_any(srv, 10, ctypes.byref(rid), ctypes.byref(status), ctypes.byref(lat),
                                       None, 0) == _lib.QTX_E_TIMEOUT
    finally:
        assert lib.qtx_server_destroy(srv) == 0



def test_native_server_groups_waiting_small_requests():
    """One slot, busy with a b=128 request while five small ones arrive: the
    three b=32 requests then run in one grouped launch, the b=16 one in
    another, each with its own status (one of the b=32 requests cannot
    converge in one Sancho-Rubio iteration) and results equal to the grouped
    solve of the request alone."""
    lib, srv = _server(slots=1, group=64)
    specs = [(24, 128, 48, 200), (5, 32, 9, 200), (7, 32, 6, 1), (3, 16, 5, 200), (4, 32, 11, 200),
             (6, 16, 4, 200)]
    keep, ids = [], []
    try:
        for i, (nb, b, ne, max_it) in enumerate(specs):
            d = make_device(num_blocks=nb, block_size=b, num_energies=ne, seed=60 + i)
            d.sr_max_iter = max_it
            h_diag = torch.from_numpy(d.h_diag).cuda()
            h_upper = torch.from_numpy(d.h_upper).cuda()
            e = torch.from_numpy(d.energies).cuda()
            out = allocate_outputs(nb, b, ne, KEYS, torch.cuda.current_device())
            keep.append((d, out, h_diag, h_upper, e))
        torch.cuda.synchronize()
        for d, out, h_diag, h_upper, e in keep:
            p, o = _problem(d, h_diag, h_upper, e, 64), _outputs(out)
            keep[len(ids)] += (p, o)
            rid = ctypes.c_int64()
            assert lib.qtx_server_submit(srv, ctypes.byref(p), ctypes.byref(o), _lib.QTX_PREC_FP64, 0,
                                         ctypes.byref(rid)) == _lib.QTX_OK
            ids.append(rid.value)
        statuses = []
        for rid in ids:
            status, lat = ctypes.c_int32(), ctypes.c_double()
            assert lib.qtx_server_wait(srv, rid, -1, ctypes.byref(status), ctypes.byref(lat), None, 0) == 0
            statuses.append(status.value)
        stats = _lib.ServerStats()
        assert lib.qtx_server_get_stats(srv, ctypes.byref(stats)) == 0
    finally:
        assert lib.qtx_server_destroy(srv) == 0
    assert statuses == [_lib.QTX_OK, _lib.QTX_OK, _lib.QTX_E_NOT_CONVERGED, _lib.QTX_OK, _lib.QTX_OK, _lib.QTX_OK]
    assert stats.grouped_launches == 2 and stats.grouped_requests == 5
    assert stats.completed == 6 and stats.failed == 0
    for (d, out, *_), (nb, b, ne, max_it) in zip(keep, specs):
        if b > 64:
            ref = TransportSolver(d, max_batch_size=64).solve(d.energies, keys=KEYS)
        else:
            with pytest.warns(RuntimeWarning) if max_it == 1 else _nullcontext():
                ref = solve_grouped([d], [d.energies], keys=KEYS)[0]
        for k in KEYS:
            assert torch.equal(out[k], ref[k]), (b, k)


def test_transport_server_shrinks_calls_to_its_budget():
    """A request whose tuned call size does not fit the server's budget runs
    in smaller calls (halved until one call's work space fits) instead of
    being refused; the observables equal a direct solve."""
    from quatrex_b200.serving import TransportServer

    class _FixedTuner:
        def best(self, b, ne, precision):
            return {"energies_per_call": 16, "gemm_path": "fp64"}

    d = make_device(num_blocks=6, block_size=32, num_energies=16, seed=8)
    lib = _lib.load()
    budget = lib.qtx_transport_footprint(6, 32, 4, _lib.QTX_PREC_FP64)
    assert lib.qtx_transport_footprint(6, 32, 16, _lib.QTX_PREC_FP64) > budget
    server = TransportServer(slots=1, memory_budget=budget, tuner=_FixedTuner(), group_small=False)
    try:
        res = server.submit(d, d.energies).result()
    finally:
        server.close()
    ref = TransportSolver(d, max_batch_size=4).solve(d.energies, keys=("density", "transmission"))
    for k in ("density", "transmission"):
        got = res[k] if not isinstance(res[k], torch.Tensor) else res[k].cpu().numpy()
        want = ref[k].cpu().numpy()
        assert abs(got - want).max() <= 1e-12 * max(abs(want).max(), 1.0), k
