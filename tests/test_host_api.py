"""Host side of the product library, run without a GPU: the arrays it builds in
the MONOLIS struct (pattern, CSC, assembly, Dirichlet) are bit-identical to
the oracle's, its parameter handling matches the reference, and it exports
every function include/*.h declares."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import problems as P
from helpers import bits_equal

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("monolis.h", "monolis_utils.h", "monolis_b200.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:void|int|void\s*\*)\s*\**\s*(monolis\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return names


def test_exports_every_declared_symbol(product):
    names = declared_functions()
    assert len(names) > 60
    missing = [n for n in names if not hasattr(product.dll, n)]
    assert not missing, missing


def test_struct_sizes_match_reference_layout(product):
    # MONOLIS_PRM: 3 x char[1024] + int[100] + double[100] (wrapper/define/monolis_def_solver_prm_c.h:148-154)
    assert C.sizeof(api.MONOLIS_PRM) == 3 * 1024 + 400 + 800
    # MONOLIS_MAT: 3 ints, 3 pointers, 6+6+4+2+3 pointers
    assert C.sizeof(api.MONOLIS_MAT) == 16 + 8 * (3 + 6 + 6 + 4 + 2 + 3)


def test_prm_defaults(product, oracle):
    # wrapper/define/monolis_def_solver_prm_c.c:7-43
    for lib in (product, oracle):
        m = api.Monolis(lib)
        I, R = m.Iarray, m.Rarray
        assert (I[1], I[2], I[3], I[4], I[5]) == (1, 1, 1000, 0, -1)
        assert (I[10], I[16], I[20], I[21], I[22], I[24]) == (1, 1, 1, 1, 1, 4)
        assert R[1] == 1e-8
        assert m.s.prm.com_part_dir_name == b"parted.0"


@pytest.mark.parametrize("problem,kw", [
    ("laplacian", dict(n=7)),
    ("elasticity", dict(n=5)),
    ("convection_diffusion", dict(n=6, peclet=50.0)),
    ("diffusion_kappa", dict(n=6)),
])
def test_assembly_bit_identical(product, oracle, problem, kw):
    builder = {"laplacian": P.laplacian, "elasticity": P.elasticity,
               "convection_diffusion": P.convection_diffusion, "diffusion_kappa": P.diffusion_kappa}[problem]
    mp, mo = api.Monolis(product), api.Monolis(oracle)
    bp, bo = builder(mp, **kw), builder(mo, **kw)
    if isinstance(bp, tuple):
        bp, bo = bp[0], bo[0]
    for f in ("csr_index", "csr_item", "csc_index", "csc_item", "csc_perm"):
        assert np.array_equal(getattr(mp, f)(), getattr(mo, f)()), f
    assert bits_equal(mp.values(), mo.values())
    assert bits_equal(bp, bo)  # Dirichlet moves columns into b identically


def test_int_star_star_pattern_matches_flat(product):
    elem = P.hex_elements(4)
    a, b = api.Monolis(product), api.Monolis(product)
    a.get_nonzero_pattern_by_simple_mesh(64, 8, 3, elem)
    b.get_nonzero_pattern_flat(64, 8, 3, elem)
    assert np.array_equal(a.csr_index(), b.csr_index()) and np.array_equal(a.csr_item(), b.csr_item())


def test_add_matrix_equals_add_elements(product, oracle):
    """Per-element add_matrix calls and the bulk entry point (row-split
    threads) give the same bits, also with repeated elements."""
    rng = np.random.default_rng(1)
    elem = P.hex_elements(5)
    elem = np.concatenate([elem, elem[::3]])  # overlap: entries get several contributions
    vals = rng.standard_normal((len(elem), 24 * 24))
    outs = []
    for lib, bulk in ((product, True), (product, False), (oracle, False)):
        m = api.Monolis(lib)
        m.get_nonzero_pattern_flat(125, 8, 3, elem)
        if bulk:
            m.add_elements(elem, 8, vals.reshape(-1), 24 * 24)
        else:
            for e in range(len(elem)):
                m.add_matrix(elem[e], vals[e].reshape(24, 24))
        outs.append(m.values().copy())
    assert bits_equal(outs[0], outs[1]) and bits_equal(outs[1], outs[2])


def test_nodal_graph_and_bcsr(product, oracle):
    # monolis_get_nonzero_pattern_by_nodal_graph_R and monolis_set_matrix_BCSR_R
    index = np.array([0, 2, 3, 5, 6], dtype=np.int32)
    item = np.array([3, 1, 0, 3, 1, 2], dtype=np.int32)
    got = []
    for lib in (product, oracle):
        m = api.Monolis(lib)
        m.get_nonzero_pattern_by_nodal_graph(4, 2, index, item)
        got.append((m.csr_index().copy(), m.csr_item().copy(), m.csc_perm().copy()))
    for k in range(3):
        assert np.array_equal(got[0][k], got[1][k])
    A = np.arange(8 * 4, dtype=np.float64)
    idx = np.array([0, 2, 4, 6, 8], dtype=np.int32)
    it = np.array([0, 1, 0, 1, 2, 3, 2, 3], dtype=np.int32)
    for lib in (product, oracle):
        m = api.Monolis(lib)
        m.set_matrix_BCSR(4, 4, 2, 8, A, idx, it)
        assert np.array_equal(m.csr_item(), it + 1)
        assert bits_equal(m.values(), A)
        v, found = m.get_scalar(2, 3, 1, 0)
        assert found and v == A[4 * 5 + 2]


def test_scalar_get_missing_entry(product):
    m = api.Monolis(product)
    elem = np.array([[0, 1], [1, 2]], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(3, 2, 1, elem)
    v, found = m.get_scalar(0, 2, 0, 0)
    assert not found and v == 0.0


def test_matrix_version_bumps(product):
    m = api.Monolis(product)
    elem = np.array([[0, 1]], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(2, 2, 1, elem)
    v0 = m.Iarray[api.B200_PRM_I_MATRIX_VERSION]
    m.add_scalar(0, 1, 0, 0, 1.0)
    b = np.zeros(2)
    m.set_Dirichlet_bc(b, 0, 0, 0.0)
    assert m.Iarray[api.B200_PRM_I_MATRIX_VERSION] == v0 + 2


def test_unsupported_method_reports_status(product):
    m = api.Monolis(product)
    elem = np.array([[0, 1]], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(2, 2, 1, elem)
    m.quiet()
    m.set_method(4)  # PipeCR: not provided
    x = np.zeros(2)
    m.solve(np.ones(2), x)
    assert m.get_error_tag() == 5 and np.all(x == 0.0)
    m.set_method(api.ITER_PIPECG)  # provided in FP64 only
    m.set_precision(1)
    m.solve(np.ones(2), x)
    assert m.get_error_tag() == 5 and np.all(x == 0.0)


def test_set_precision_validates(product):
    m = api.Monolis(product)
    with pytest.raises(ValueError):
        m.set_precision(7)
