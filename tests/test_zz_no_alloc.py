"""The allocation-free inner product (monolis_b200_inner_product_noalloc_R)
against an independent host sum (math.fsum of the exact products) and the
library's regular inner product (monolis_inner_product_R).

The no-alloc entry point is for callers that cannot call cudaMalloc when they
need a dot product (an application that keeps all device memory in its own
pool, a loop that must not take cudaMalloc's implicit synchronisation); its
reduction scratch is a fixed array inside the library. This file is named so
that pytest collects it last; it also passes on its own in a fresh process.
"""
import ctypes as C
import math
from fractions import Fraction

import numpy as np
import pytest

from monolis_b200 import api

pytestmark = pytest.mark.gpu

MAX_N = 16384 * 256 * 4  # capacity stated in include/monolis_b200.h


def _regular_dot(lib, x, y):
    # the existing entry point works on the vectors of a MONOLIS struct of N rows
    n = len(x)
    m = api.Monolis(lib)
    idx = np.arange(n + 1, dtype=np.int32)
    item = np.arange(n, dtype=np.int32)
    m.set_matrix_BCSR(n, n, 1, n, np.ones(n), idx, item)
    s = m.inner_product(1, x, y)
    m.finalize()
    return s


def _exact_dot(x, y):
    """The dot product rounded once: each product taken exactly (a rational
    number), split into two doubles (its rounding and the remainder, which
    is exact: a product of two doubles has at most 106 significant bits),
    and all of them summed exactly by math.fsum."""
    terms = []
    for a, b in zip(x.tolist(), y.tolist()):
        p = Fraction(a) * Fraction(b)
        hi = float(p)
        terms.append(hi)
        terms.append(float(p - Fraction(hi)))
    return math.fsum(terms)


def _noalloc(lib, n, d_x, d_y, stream):
    import torch

    d_out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    rc = lib.monolis_b200_inner_product_noalloc_R(n, C.c_void_p(d_x.data_ptr()), C.c_void_p(d_y.data_ptr()),
                                                 C.c_void_p(d_out.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == 0
    stream.synchronize()
    return d_out.item()


def test_noalloc_inner_product_matches_regular(gpu):
    import torch

    lib = gpu
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(2024)
    n = 200_003
    for call in range(2):  # two calls in a row share the same device scratch
        x = rng.standard_normal(n)
        y = rng.standard_normal(n) + (0.5 if call else 0.0)
        exact = _exact_dot(x, y)
        ref = _regular_dot(lib, x, y)
        got = _noalloc(lib, n, torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), stream)
        # a tree of FP64 sums: within 1e-13 of sum |x_i y_i| of the exact value
        scale = float(np.abs(x * y).sum())
        assert abs(got - exact) <= 1e-13 * scale, (call, got, exact)
        assert abs(got - ref) <= 1e-13 * scale, (call, got, ref)


def test_noalloc_empty_and_full_capacity(gpu):
    """n = 0 gives 0 (the result is still written); n at the stated maximum
    runs, checked against a numpy sum of the same products."""
    import torch

    stream = torch.cuda.current_stream()
    d = torch.ones(1, dtype=torch.float64, device="cuda")
    assert _noalloc(gpu, 0, d, d, stream) == 0.0
    rng = np.random.default_rng(7)
    x = rng.standard_normal(MAX_N)
    y = rng.standard_normal(MAX_N)
    ref = float(np.dot(x, y))
    for _ in range(2):
        got = _noalloc(gpu, MAX_N, torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda(), stream)
        assert abs(got - ref) <= 1e-12 * float(np.abs(x * y).sum()), (got, ref)


def test_noalloc_rejects_oversize(gpu):
    import torch

    d = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = gpu.monolis_b200_inner_product_noalloc_R(MAX_N + 1, C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
                                                 C.c_void_p(d.data_ptr()), None)
    assert rc == 5  # MONOLIS_B200_BAD_INPUT, nothing launched
