"""The allocation-free binning entry point (psum_bin_positions_noalloc).

Callers that cannot call cudaMalloc (device memory owned by another
runtime's pool, or a loop under a fixed memory budget) bin their own device
positions with scratch that lives in a fixed device array inside the
library.  Its results must equal those of the allocating entry point
(psum_pic_bin, context-based) exactly, on consecutive calls that reuse the
shared scratch.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import psum_b200 as P

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def reference_bin(cells, lo, hi, pos):
    """psum_pic_bin through a context (FP64 positions, loaded as given)."""
    n = pos.shape[1]
    ctx = P.ParticleContext(cells, lo, hi, (0,) * len(cells), P.FP64)
    sp = ctx.add_species(1.0, 1.0, 1.0, n)
    ctx.load(sp, pos, np.zeros((3, n)))
    ncell = int(np.prod(cells))
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    counts = torch.zeros(ncell, dtype=torch.int64, device="cuda")
    offs = torch.zeros(ncell, dtype=torch.int64, device="cuda")
    perm = torch.zeros(n, dtype=torch.int64, device="cuda")
    m = ctx.bin(sp, keys, counts, offs, perm)
    torch.cuda.synchronize()
    out = (keys.cpu().numpy(), counts.cpu().numpy(), offs.cpu().numpy(), perm.cpu().numpy()[:m], m)
    ctx.close()
    return out


def noalloc_bin(cells, lo, hi, pos_dev):
    g = P._lib.GridDesc()
    g.dim = len(cells)
    for a in range(3):
        g.cells[a] = cells[a] if a < g.dim else 1
        g.lower[a] = lo[a] if a < g.dim else 0.0
        g.upper[a] = hi[a] if a < g.dim else 1.0
    n = pos_dev.shape[1]
    ncell = int(np.prod(cells))
    keys = torch.full((n,), -7, dtype=torch.int64, device="cuda")
    counts = torch.full((ncell,), 7, dtype=torch.int64, device="cuda")
    offs = torch.full((ncell,), 7, dtype=torch.int64, device="cuda")
    perm = torch.full((n,), 7, dtype=torch.int64, device="cuda")
    m = C.c_ulonglong()
    torch.cuda.synchronize()
    P.check(P.lib().psum_bin_positions_noalloc(C.byref(g), n, pos_dev.data_ptr(), keys.data_ptr(), counts.data_ptr(),
                                               offs.data_ptr(), perm.data_ptr(), C.byref(m), None))
    return keys.cpu().numpy(), counts.cpu().numpy(), offs.cpu().numpy(), perm.cpu().numpy()[:m.value], m.value


@pytest.mark.parametrize("case", ["2d", "3d"])
def test_noalloc_bin_matches_allocating_entry_point_twice(case):
    rng = np.random.default_rng(77)
    if case == "2d":
        cells, lo, hi = (300, 200), (0.0, -1.0), (3.0, 1.0)
    else:
        cells, lo, hi = (40, 30, 20), (0.0, 0.0, 0.0), (4.0, 3.0, 2.0)
    for call in range(2):            # two calls in a row share the scratch array
        n = 200000 - 37 * call       # a different size on the second call
        pos = np.stack([rng.uniform(l - 0.1 * (h - l), h + 0.1 * (h - l), n) for l, h in zip(lo, hi)])
        pos[0, ::101] = np.nan       # invalid particles are not in the grid
        exp = reference_bin(cells, lo, hi, pos)
        got = noalloc_bin(cells, lo, hi, torch.tensor(pos, device="cuda"))
        assert got[4] == exp[4]
        for g_, e_ in zip(got[:4], exp[:4]):
            assert g_.shape == e_.shape
            assert (g_ == e_).all()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    g = P._lib.GridDesc()
    g.dim = 2
    g.cells[0], g.cells[1], g.cells[2] = 8, 8, 1
    g.upper[0] = g.upper[1] = g.upper[2] = 1.0
    big = torch.zeros((2, (1 << 18) + 1), dtype=torch.float64, device="cuda")
    out = torch.zeros((1 << 18) + 1, dtype=torch.int64, device="cuda")
    m = C.c_ulonglong()
    code = P.lib().psum_bin_positions_noalloc(C.byref(g), big.shape[1], big.data_ptr(), out.data_ptr(),
                                              out.data_ptr(), out.data_ptr(), out.data_ptr(), C.byref(m), None)
    assert code == 1 and b"exceeds" in P.lib().psum_last_error()
    # a count of 2^63 or more must not pass the limit as a negative signed value
    code = P.lib().psum_bin_positions_noalloc(C.byref(g), (1 << 63) + 5, big.data_ptr(), out.data_ptr(),
                                              out.data_ptr(), out.data_ptr(), out.data_ptr(), C.byref(m), None)
    assert code == 1 and b"exceeds" in P.lib().psum_last_error()
    g.cells[0] = g.cells[1] = 2048          # 4,194,304 cells > the 1,048,576-cell limit
    code = P.lib().psum_bin_positions_noalloc(C.byref(g), 10, big.data_ptr(), out.data_ptr(), out.data_ptr(),
                                              out.data_ptr(), out.data_ptr(), C.byref(m), None)
    assert code == 1 and b"exceed" in P.lib().psum_last_error()
    # factors whose product overflows 64 bits are refused factor by factor
    g.dim = 3
    g.cells[0] = g.cells[1] = g.cells[2] = (1 << 31) - 1
    code = P.lib().psum_bin_positions_noalloc(C.byref(g), 10, big.data_ptr(), out.data_ptr(), out.data_ptr(),
                                              out.data_ptr(), out.data_ptr(), C.byref(m), None)
    assert code == 1 and b"exceed" in P.lib().psum_last_error()


def test_noalloc_allocates_no_device_memory():
    """After a warm-up call, further calls leave the device's free memory unchanged."""
    cells, lo, hi = (300, 200), (0.0, -1.0), (3.0, 1.0)
    rng = np.random.default_rng(5)
    pos = torch.tensor(np.stack([rng.uniform(l, h, 100000) for l, h in zip(lo, hi)]), device="cuda")
    first = noalloc_bin(cells, lo, hi, pos)           # warm-up: module load and symbol look-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    again = noalloc_bin(cells, lo, hi, pos)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # the outputs of noalloc_bin are allocated by the test before the call; they come from torch's cache, so
    # the free memory the driver reports does not change unless the library allocates
    assert torch.cuda.memory_reserved() == reserved0
    assert free1 == free0
    for a, b in zip(first, again):
        assert np.array_equal(np.asarray(a), np.asarray(b))


def test_noalloc_clamps_positions_just_below_the_upper_bound():
    """A position one ulp below `upper` whose (p - lo) * dr truncates to `cells` bins into the last cell."""
    from oracle import oracle as O
    cells, lo, hi = (199, 300), (0.0, 0.0), (3.3, 3.0)
    n = 1000
    rng = np.random.default_rng(9)
    pos = np.stack([rng.uniform(lo[a], hi[a], n) for a in range(2)])
    edge = [np.nextafter(hi[a], lo[a]) for a in range(2)]
    pos[0, ::7] = edge[0]
    pos[1, ::5] = edge[1]
    dr = [1.0 / ((hi[a] - lo[a]) / cells[a]) for a in range(2)]
    assert any(int((edge[a] - lo[a]) * dr[a]) == cells[a] for a in range(2))   # the case is reached
    got = noalloc_bin(cells, lo, hi, torch.tensor(pos, device="cuda"))
    ek, ec, eo, ep = O.bin_particles(O.make_grid(cells, lo, hi, (0, 0)), pos)
    assert got[0].max() < cells[0] * cells[1]
    assert np.array_equal(got[0], ek) and np.array_equal(got[1], ec.astype(np.int64))
    assert np.array_equal(got[2], eo.astype(np.int64)) and np.array_equal(got[3], ep.astype(np.int64))
