"""CPU checks of the matvec-form autotuner's table logic (autotune.py):
size buckets, lookups by dims and rows, the library default where the table
has no entry, and make_options(pass_kernel="auto") resolved per call."""

import numpy as np


def test_buckets_and_lookup(pkg):
    import importlib
    at = importlib.import_module(pkg.__name__ + ".autotune")
    assert [at.bucket_of(n) for n in (1, 9_999, 10_000, 99_999, 3_000_000, 10**9)] == [4, 4, 4, 4, 6, 7]
    table = {"classes": {"dims2_b5": {"pass_kernel": 3}, "dims3_b6": {"pass_kernel": 2}}}
    assert at.choose_pass_kernel(2, 300_000, table) == 3
    assert at.choose_pass_kernel(3, 2_000_000, table) == 2
    assert at.choose_pass_kernel(4, 2_000_000, table) == 2  # 4+ dims use the 3-dim classes
    assert at.choose_pass_kernel(2, 50_000_000, table) == 0  # no entry: the library's default
    assert at.choose_pass_kernel(3, 300_000, {}) == 0


def test_auto_option_is_resolved_per_call(pkg):
    import importlib
    ab = importlib.import_module(pkg.__name__ + ".absorber")
    at = importlib.import_module(pkg.__name__ + ".autotune")
    o = pkg.make_options(tol=1e-8, pass_kernel="auto")
    assert o.pass_kernel == ab.PASS_KERNEL_AUTO
    for dims, n in ((2, 40_000), (3, 3_000_000), (3, 50_000_000)):
        r = ab._resolve_options(o, dims, n)
        assert r.pass_kernel == at.choose_pass_kernel(dims, n) and r.pass_kernel in (0, 1, 2, 3)
        assert r.tol == o.tol and o.pass_kernel == ab.PASS_KERNEL_AUTO  # a copy; o untouched
    fixed = pkg.make_options(pass_kernel=2)
    assert ab._resolve_options(fixed, 3, 10) is fixed
    assert np.isfinite(o.tol)
