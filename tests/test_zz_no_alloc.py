"""The allocation-free entry point b200fe_demean_sorted_noalloc.

It serves callers that cannot allocate device memory while they use this
library (a host application that keeps all device memory in its own pool, or
a plugin that must not grow its CUDA footprint mid-session); its only scratch
is a fixed array inside the library, shared by every call and keeping the
last call's contents.  This file is collected last, so a run that stops at
the first failure has already run every other test, and it must pass both
alone in a fresh process and after the other tests.

Checked through the C ABI: two calls in a row give the same within transform
as the regular absorber (b200fe_absorb_device with one FE dimension) and as
group means computed in numpy, within the relative tolerance of the other
parity tests, unweighted and weighted; the second call leaves the device's
free memory unchanged; oversized, unsorted, negative and out-of-range ids are
rejected.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL_TOL = 1e-8  # the bar of tests/test_gpu_parity.py


def _sorted_panel(panels, seed):
    p = panels.akm_two_way(40_000, n_firms=800, seed=seed, three_way=False)
    p = panels.subset(p, panels.drop_singletons(p.fes))
    order = np.argsort(p.fes[0], kind="stable")  # rows ordered by worker
    g = np.ascontiguousarray(p.fes[0][order])
    V = np.ascontiguousarray(np.column_stack([p.y, p.X])[order].T)  # (cols, n): column-major
    return g, V, int(g.max()) + 1


@pytest.mark.parametrize("weighted", [False, True])
def test_noalloc_matches_absorber_on_two_calls(pkg, libmod, panels, weighted):
    import torch

    lib = libmod.load()
    g, V, G = _sorted_panel(panels, seed=41 if weighted else 43)
    cols, n = V.shape
    dv = torch.from_numpy(V).cuda()
    dg = torch.from_numpy(g).cuda()
    w = np.random.default_rng(7).lognormal(0.0, 0.5, size=n) if weighted else None
    dw = torch.from_numpy(w).cuda() if weighted else None
    ab = pkg.Absorber(0)
    try:
        ref, r = ab.absorb_device(dv, [dg], [G], dw, pkg.make_options(tol=1e-10))
        assert r.status == libmod.OK
        ref = ref.cpu().numpy()
    finally:
        ab.close()
    scale = np.linalg.norm(V, axis=1)
    # the one-way within transform directly: v minus its weighted group mean
    ww = w if weighted else np.ones(n)
    W = np.bincount(g, weights=ww, minlength=G)
    direct = np.empty_like(V)
    for c in range(cols):
        m = np.bincount(g, weights=ww * V[c], minlength=G) / np.where(W > 0, W, 1.0)
        direct[c] = V[c] - m[g]
    bufs = [torch.empty_like(dv) for _ in range(2)]  # no allocation between the calls
    torch.cuda.synchronize()
    free = []
    for out in bufs:
        rc = lib.b200fe_demean_sorted_noalloc(
            dv.data_ptr(), n, cols, dg.data_ptr(), G, dw.data_ptr() if weighted else None,
            out.data_ptr(), None)
        torch.cuda.synchronize()
        assert rc == libmod.OK
        free.append(torch.cuda.mem_get_info()[0])
    assert free[1] == free[0]  # a repeated call places nothing on the device
    outs = [b.cpu().numpy() for b in bufs]
    for o in outs:
        err = float((np.linalg.norm(o - ref, axis=1) / scale).max())
        assert err <= REL_TOL, err
        err_direct = float((np.linalg.norm(o - direct, axis=1) / scale).max())
        assert err_direct <= REL_TOL, err_direct
    assert np.array_equal(outs[0], outs[1])


def test_noalloc_rejects_oversized_and_unsorted(libmod):
    import torch

    lib = libmod.load()
    n = 1000
    dv = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    out = torch.empty_like(dv)
    g_sorted = (torch.arange(n, dtype=torch.int32, device="cuda") // 10).contiguous()
    rc = lib.b200fe_demean_sorted_noalloc(dv.data_ptr(), n, 1, g_sorted.data_ptr(), (1 << 20) + 1,
                                          None, out.data_ptr(), None)
    assert rc == libmod.INVALID_ARG
    g_unsorted = torch.flip(g_sorted, [0]).contiguous()
    rc = lib.b200fe_demean_sorted_noalloc(dv.data_ptr(), n, 1, g_unsorted.data_ptr(), 100, None,
                                          out.data_ptr(), None)
    assert rc == libmod.INVALID_ARG


def test_noalloc_rejects_negative_and_out_of_range_ids(libmod):
    import torch

    lib = libmod.load()
    n = 1000
    dv = torch.zeros((1, n), dtype=torch.float64, device="cuda")
    out = torch.empty_like(dv)
    g = (torch.arange(n, dtype=torch.int32, device="cuda") // 10).contiguous()  # 0..99
    g_neg = g.clone()
    g_neg[0] = -1  # still non-decreasing, one negative id
    rc = lib.b200fe_demean_sorted_noalloc(dv.data_ptr(), n, 1, g_neg.data_ptr(), 100, None,
                                          out.data_ptr(), None)
    assert rc == libmod.INVALID_ARG
    g_big = g.clone()
    g_big[-1] = 100  # == num_groups
    rc = lib.b200fe_demean_sorted_noalloc(dv.data_ptr(), n, 1, g_big.data_ptr(), 100, None,
                                          out.data_ptr(), None)
    assert rc == libmod.INVALID_ARG
    # a valid call right after the rejections starts from a cleared status word
    rc = lib.b200fe_demean_sorted_noalloc(dv.data_ptr(), n, 1, g.data_ptr(), 100, None,
                                          out.data_ptr(), None)
    torch.cuda.synchronize()
    assert rc == libmod.OK
