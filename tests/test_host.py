"""Host-side logic that needs no GPU: library exports, block maps, batching."""

import ctypes
import os
import re

import numpy as np
import pytest
from scipy import sparse

from quatrex_b200 import _lib
from quatrex_b200.datastructures import DSDBCOO, block_sort_index, btd_layout_from_coords

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

def _header_symbols():
    text = open(os.path.join(ROOT, "include", "qtx_rgf.h")).read()
    return sorted(set(re.findall(r"^\s*(?:qtx_status|const char\*|int64_t|size_t)\s+(qtx_\w+)\s*\(", text, re.M)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    names = _header_symbols()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, n
    assert set(_lib.SIGNATURES) == set(names)
    assert b"sm_100a" in lib.qtx_version()


def test_library_without_device_reports_error():
    lib = _lib.load()
    p = ctypes.c_void_p()
    # on a machine without a usable CUDA device the context cannot be created
    st = lib.qtx_ctx_create(0, ctypes.byref(p))
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if not has_gpu:
        assert st != _lib.QTX_OK
    else:
        assert st == _lib.QTX_OK
        lib.qtx_ctx_destroy(p)


def _bt_pattern(sizes, density, rng):
    offs = np.hstack(([0], np.cumsum(sizes)))
    n = offs[-1]
    a = np.zeros((n, n), dtype=np.complex128)
    for i in range(len(sizes)):
        for j in range(max(0, i - 1), min(len(sizes), i + 2)):
            blk = (rng.random((sizes[i], sizes[j])) < density) * (rng.standard_normal((sizes[i], sizes[j])) + 1j)
            a[offs[i]:offs[i + 1], offs[j]:offs[j + 1]] = blk
    return a


@pytest.mark.parametrize("sizes", [[2] * 10, [2, 2, 2, 4, 4, 2, 2, 2], [5, 3, 7]])
@pytest.mark.parametrize("density", [0.5, 1.0])
def test_layout_roundtrip(sizes, density):
    rng = np.random.default_rng(1)
    dense = _bt_pattern(sizes, density, rng)
    m = DSDBCOO.from_sparray(sparse.coo_matrix(dense), np.array(sizes), (3,))
    assert np.allclose(m.to_dense()[1], dense)
    lay = m.layout
    nb = len(sizes)
    offs = np.hstack(([0], np.cumsum(sizes)))
    for i in range(nb):
        for j in range(max(0, i - 1), min(nb, i + 2)):
            k = 2 * i + j
            blk = m.blocks[i, j][0]
            assert np.allclose(blk, dense[offs[i]:offs[i + 1], offs[j]:offs[j + 1]])
            if density == 1.0:
                assert lay.local_index[k] is None  # dense row-major slice, read in place
    # blocks are contiguous and in (0,0),(0,1),(1,0),(1,1),... order
    starts = [s for s in lay.block_offset if s >= 0]
    assert starts == sorted(starts)


def test_layout_rejects_non_btd():
    rows = np.array([0, 5])
    cols = np.array([5, 0])
    with pytest.raises(ValueError):
        btd_layout_from_coords(rows, cols, [2, 2, 2])


def test_block_sort_matches_upstream_rule():
    # upstream: block row by block row, inside a block row by block column,
    # stable inside a block (compute_block_sort_index)
    rows = np.array([0, 0, 1, 2, 2, 3, 3])
    cols = np.array([0, 2, 1, 0, 3, 2, 3])
    order = block_sort_index(rows, cols, [2, 2])
    assert list(zip(rows[order], cols[order])) == [(0, 0), (1, 1), (0, 2), (2, 0), (2, 3), (3, 2), (3, 3)]


def test_set_get_block_and_zeros_like():
    dense = _bt_pattern([3, 3, 3], 1.0, np.random.default_rng(2))
    m = DSDBCOO.from_sparray(sparse.coo_matrix(dense), np.array([3, 3, 3]), (4,))
    z = DSDBCOO.zeros_like(m)
    assert np.all(z.to_dense() == 0)
    val = np.arange(9).reshape(3, 3) * (1 + 1j)
    z.blocks[1, 2] = val
    assert np.allclose(z.blocks[1, 2], val)
    assert np.allclose(z.to_dense()[2][3:6, 6:9], val)


def test_transport_footprint_is_host_arithmetic():
    """Admission footprint of one transport call: grows with the energies per
    call and with the slice buffers of the mixed form; invalid shapes give 0."""
    lib = _lib.load()
    f8 = lib.qtx_transport_footprint(16, 64, 8, _lib.QTX_PREC_FP64)
    f16 = lib.qtx_transport_footprint(16, 64, 16, _lib.QTX_PREC_FP64)
    m16 = lib.qtx_transport_footprint(16, 64, 16, _lib.QTX_PREC_MIXED)
    assert 0 < f8 < f16 < m16
    # the recursion state alone: 3 nb + 20 block stacks of 16 b^2 bytes per energy
    assert f16 - f8 >= 8 * (3 * 16 + 20) * 16 * 64 * 64
    assert lib.qtx_transport_footprint(1, 64, 8, _lib.QTX_PREC_FP64) == 0


def test_serving_call_size_fits_the_budget():
    """A request's energies per call: the tuned size capped by the request's
    energies, halved until one call's footprint fits the server budget; one
    energy per call is the floor (the native server refuses the rest)."""
    from quatrex_b200.serving import call_size

    lib = _lib.load()
    fp = lambda ne, prec="fp64": lib.qtx_transport_footprint(64, 256, ne, _lib.QTX_PREC_FP64 if prec == "fp64"
                                                             else _lib.QTX_PREC_MIXED)
    assert call_size(lib, 64, 256, 1024, 148, "fp64", 10 ** 15) == 148
    assert call_size(lib, 64, 256, 20, 148, "fp64", 10 ** 15) == 20
    budget = fp(40)
    got = call_size(lib, 64, 256, 1024, 148, "fp64", budget)
    assert got == 37 and fp(got) <= budget < fp(2 * got)  # 148 -> 74 -> 37
    assert call_size(lib, 64, 256, 1024, 148, "mixed", fp(37)) <= 37
    assert call_size(lib, 64, 256, 1024, 148, "fp64", 1) == 1


def test_grouped_footprint_is_host_arithmetic():
    """Work space of a grouped launch: one (3 nb_max + 20)-block work space per
    resident CTA (never more CTAs than pairs), plus descriptors; block sizes
    above 64 are not offered (0)."""
    from quatrex_b200.transport import grouped_footprint_bytes

    one = grouped_footprint_bytes([8], [1], 32)
    assert one >= (3 * 8 + 20) * 16 * 32 * 32
    # a longer device raises the per-CTA work space, more energies more CTAs
    assert grouped_footprint_bytes([16], [1], 32) > one
    assert grouped_footprint_bytes([8], [4], 32) > one
    # the work space follows the longest device of the group
    mixed = grouped_footprint_bytes([8, 16], [2, 2], 32)
    assert mixed >= 4 * (3 * 16 + 20) * 16 * 32 * 32
    assert grouped_footprint_bytes([8], [4], 64) > grouped_footprint_bytes([8], [4], 32)
    assert grouped_footprint_bytes([8], [4], 65) == 0
    assert grouped_footprint_bytes([8], [0], 32) == 0


def test_peak_mask_matches_upstream_filter():
    """quatrex_b200.transport.peak_mask (torch) picks the energies that upstream
    ElectronSolver._filter_peaks zeroes (fixture written by the upstream code)."""
    import torch

    from oracle import rgf_oracle as orc
    from quatrex_b200.transport import filter_peaks, peak_mask

    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "observables_small.npz"))
    dos = torch.from_numpy(g["dos"])
    mask = peak_mask(dos, g["energies"], float(g["peak_limit"]))
    assert np.array_equal(mask.numpy(), g["peak_mask"])
    assert np.array_equal(mask.numpy(), orc.peak_mask(g["dos"], g["energies"], float(g["peak_limit"])))
    # uneven spacing follows numpy.gradient too
    e = np.sort(np.random.default_rng(0).uniform(-2, 2, 40))
    got = torch.gradient(dos, spacing=(torch.from_numpy(e),), dim=0)[0].numpy()
    assert np.allclose(got, np.gradient(g["dos"], e, axis=0), rtol=1e-12, atol=0)
    out = {"density": torch.ones(40, 5), "dos": dos.clone(), "gl_diag": torch.ones(40, 5, 2, 2)}
    filter_peaks(out, mask)
    assert (out["density"][mask] == 0).all() and (out["density"][~mask] == 1).all()
    assert (out["gl_diag"][mask] == 0).all() and torch.equal(out["dos"], dos)


def test_uneven_batch_job_plan():
    """BatchedTransport.jobs: one grouped job per block size <= 64, the larger
    instances one by one, every instance exactly once, longest job first; no
    grouping when it is switched off."""
    from types import SimpleNamespace

    from quatrex_b200.batching import BatchedTransport, Instance, instance_flops

    specs = [(6, 16, 8), (9, 32, 20), (4, 32, 5), (7, 64, 12), (5, 128, 9), (3, 512, 4), (8, 16, 3)]
    insts = []
    for q, (nb, b, ne) in enumerate(specs):
        d = SimpleNamespace(num_blocks=nb, block_size=b)
        insts.append(Instance(d, np.linspace(-1, 1, ne)))
    jobs = BatchedTransport.jobs(SimpleNamespace(group_small=True), insts)
    kinds = {tuple(sorted(idx)): kind for kind, idx in jobs}
    assert kinds == {(0, 6): "group", (1, 2): "group", (3,): "group", (4,): "one", (5,): "one"}
    assert sorted(i for _, idx in jobs for i in idx) == list(range(len(specs)))
    cost = [sum(instance_flops(insts[i].device, len(insts[i].energies)) for i in idx) for _, idx in jobs]
    assert cost == sorted(cost, reverse=True)
    plain = BatchedTransport.jobs(SimpleNamespace(group_small=False), insts)
    assert all(kind == "one" and len(idx) == 1 for kind, idx in plain) and len(plain) == len(specs)


def _fixture_rowptr(g, tag):
    keys, ptrs, lens = g[f"csr_{tag}_keys"], g[f"csr_{tag}_ptrs"], g[f"csr_{tag}_lens"]
    out, at = {}, 0
    for k, n in zip(keys, lens):
        out[(int(k[0]), int(k[1]))] = ptrs[at:at + n]
        at += n
    return out


@pytest.mark.parametrize("sym", [False, True], ids=["full", "symmetric"])
def test_layouts_match_upstream_fixture(sym):
    """DSDBCOO and DSDBCSR built here from the same sparse matrix hold the data
    in upstream's order, with upstream's row/column indices and row-pointer
    map (tests/golden/dsdb_layouts.npz, written by upstream from_sparray)."""
    from quatrex_b200.datastructures import DSDBCSR, layout_of

    g = np.load(os.path.join(GOLDEN, "dsdb_layouts.npz"))
    tag = "sym" if sym else "full"
    sizes = g["block_sizes"]
    coo = DSDBCOO.from_sparray(sparse.coo_matrix(g["a"]), sizes, (1,), symmetry=sym)
    assert np.array_equal(coo.rows, g[f"coo_{tag}_rows"])
    assert np.array_equal(coo.cols, g[f"coo_{tag}_cols"])
    assert np.array_equal(coo.data[0], g[f"coo_{tag}_data"])
    csr = DSDBCSR.from_sparray(sparse.coo_matrix(g["a"]), sizes, (1,), symmetry=sym)
    assert np.array_equal(csr.cols, g[f"csr_{tag}_cols"])
    assert np.array_equal(csr.data[0], g[f"csr_{tag}_data"])
    ref_map = _fixture_rowptr(g, tag)
    assert set(csr.rowptr_map) == set(ref_map)
    for k, rp in ref_map.items():
        assert np.array_equal(csr.rowptr_map[k], rp), k

    class StandIn:  # only the attributes an upstream DSDBCSR exposes
        pass

    s = StandIn()
    s.data, s.cols, s.rowptr_map, s.block_sizes = csr.data, csr.cols, ref_map, sizes
    lay_s, lay_c = layout_of(s), layout_of(coo)
    assert np.array_equal(lay_s.block_offset, lay_c.block_offset)
    assert np.array_equal(lay_s.block_nnz, lay_c.block_nnz)
    for a, b in zip(lay_s.local_index, lay_c.local_index):
        assert (a is None and b is None) or np.array_equal(a, b)


@pytest.mark.parametrize("kind", ["conj", "neg_conj", "identity"])
def test_symmetric_storage_completion(kind):
    """get_block / to_dense of symmetric storage complete the lower blocks as
    symmetry_op(X_ij^T) and the diagonal blocks as U + symmetry_op(U^T) with
    the diagonal halved, for the three operators quatrex uses."""
    from quatrex_b200.datastructures import DSDBCSR

    rng = np.random.default_rng(4)
    sizes = np.array([3, 4, 3])
    full = _bt_pattern(list(sizes), 1.0, rng)
    op = {"conj": np.conj, "neg_conj": lambda x: -np.conj(x), "identity": lambda x: x}[kind]
    m = {"conj": full + full.conj().T, "neg_conj": full - full.conj().T, "identity": full + full.T}[kind]
    for cls in (DSDBCOO, DSDBCSR):
        x = cls.from_sparray(sparse.coo_matrix(m), sizes, (2,), symmetry=True, symmetry_op=op)
        assert np.allclose(x.to_dense()[1], m)
        assert np.allclose(x.blocks[2, 1], m[7:10, 3:7])
        assert np.allclose(x.blocks[1, 1], m[3:7, 3:7])


def test_host_batched_factorisations_equal_numpy():
    """The Spectral OBC's small SVD / eig on host threads (upstream's default
    compute location) split the batch over threads with single-threaded BLAS
    and return exactly what one NumPy call returns."""
    from quatrex_b200.nevp import _host_batched

    rng = np.random.default_rng(3)
    p0 = rng.standard_normal((37, 24, 8)) + 1j * rng.standard_normal((37, 24, 8))
    u, s, vh = _host_batched(lambda x: np.linalg.svd(x, full_matrices=False), p0, 3)
    u1, s1, vh1 = np.linalg.svd(p0, full_matrices=False)
    assert np.allclose(s, s1, rtol=1e-14, atol=0)
    assert np.allclose(u @ (s[..., None] * vh), p0, rtol=0, atol=1e-12)
    a = rng.standard_normal((37, 8, 8)) + 1j * rng.standard_normal((37, 8, 8))
    w, v = _host_batched(lambda x: np.linalg.eig(x), a, 2)
    assert np.allclose(a @ v, v * w[..., None, :], atol=1e-11)


def test_autotuner_cache_and_keys(tmp_path):
    """Autotuner keys bucket the batch to a power of two; a cached choice is
    returned without measuring anything (no device needed), and the table
    survives a save/load round trip."""
    from quatrex_b200.autotune import Autotuner

    assert Autotuner.key(256, 100, "fp64") == "b256-n128-fp64"
    assert Autotuner.key(64, 148, "mixed") == "b64-n256-mixed"
    assert Autotuner.key(32, 1, "fp64") == "b32-n1-fp64"
    path = tmp_path / "sub" / "autotune.json"
    t = Autotuner(cache_path=str(path))
    choice = {"energies_per_call": 148, "gemm_path": "fp64", "graph": False, "probe_solves_per_s": 1.0}
    t.table[Autotuner.key(256, 148, "fp64")] = choice
    t.save()
    assert path.exists() and not (tmp_path / "sub" / "autotune.json.tmp").exists()
    t2 = Autotuner(cache_path=str(path))
    # 130 .. 256 energies share the bucket of 148
    assert t2.best(256, 200, "fp64") == choice
    assert t2.lookup(256, 100, "fp64") is None
