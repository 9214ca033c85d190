"""Device assembly (monolis_b200_device_add_elements_R,
monolis_b200_device_set_Dirichlet_bc_R) against the host calls made in order:
the device values and right-hand side must be bit-identical to the arrays
that monolis_add_matrix_to_sparse_matrix_R / monolis_set_Dirichlet_bc_R
produce on the host (which the host tests hold bit-identical to the oracle)."""
import ctypes as C

import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import problems as P
from helpers import bits_equal

pytestmark = pytest.mark.gpu


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def device_values(m):
    nd = m.NDOF
    out = np.empty(m.NZ * nd * nd)
    assert m.lib.monolis_b200_device_get_values(m.p, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
    return out


def mesh_problem(n, nd, seed):
    rng = np.random.default_rng(seed)
    elem = P.hex_elements(n)
    nl = 8 * nd
    shared = rng.standard_normal((nl, nl))
    per = rng.standard_normal((len(elem), nl * nl))
    scale = np.exp(rng.standard_normal(len(elem)))
    return elem, shared, per, scale


@pytest.mark.parametrize("nd", [1, 3])
@pytest.mark.parametrize("mode", ["shared", "shared_scaled", "per_element"])
def test_device_add_elements_bit_identical(gpu, nd, mode):
    import torch
    n = 6
    elem, shared, per, scale = mesh_problem(n, nd, 7 + nd)
    host = api.Monolis(gpu)
    devm = api.Monolis(gpu)
    for m in (host, devm):
        m.get_nonzero_pattern_flat(n ** 3, 8, nd, elem)
    if mode == "per_element":
        host.add_elements(elem, 8, per.reshape(-1), per.shape[1])
        args = (dev(per.reshape(-1)), per.shape[1], None)
    else:
        sc = scale if mode == "shared_scaled" else None
        host.add_elements(elem, 8, shared.reshape(-1), 0, scale=sc)
        args = (dev(shared.reshape(-1)), 0, None if sc is None else dev(sc))
    d_elem = dev(elem)
    d_val, stride, d_scale = args
    # two passes: contributions accumulate onto the existing values
    for rep in range(2):
        rc = gpu.monolis_b200_device_add_elements_R(devm.p, len(elem), 8, d_elem.data_ptr(), d_val.data_ptr(), stride,
                                                    None if d_scale is None else d_scale.data_ptr())
        assert rc == 0
    if mode == "per_element":
        host.add_elements(elem, 8, per.reshape(-1), per.shape[1])
    else:
        host.add_elements(elem, 8, shared.reshape(-1), 0, scale=scale if mode == "shared_scaled" else None)
    torch.cuda.synchronize()
    assert bits_equal(device_values(devm), host.values())


def test_device_dirichlet_bit_identical(gpu):
    """Repeated conditions, a different value the second time, non-zero
    values, interleaved order: device result = host calls in list order."""
    import torch
    n, nd = 6, 3
    elem, shared, _, scale = mesh_problem(n, nd, 3)
    rng = np.random.default_rng(11)
    host = api.Monolis(gpu)
    devm = api.Monolis(gpu)
    for m in (host, devm):
        m.get_nonzero_pattern_flat(n ** 3, 8, nd, elem)
        m.add_elements(elem, 8, shared.reshape(-1), 0, scale=scale)
    b0 = rng.standard_normal(n ** 3 * nd)
    nodes = list(range(0, n ** 3, n))[:20]
    bc = [(nd_, d, float(rng.standard_normal())) for nd_ in nodes for d in range(nd)]
    bc += [(nodes[3], 1, 2.5), (nodes[0], 0, -1.0), (37, 2, 0.75)]   # repeats and an interior dof
    rng.shuffle(bc)
    hb = b0.copy()
    for (node, d, v) in bc:
        host.set_Dirichlet_bc(hb, node, d, v)
    d_b = dev(b0)
    node_a = np.array([c[0] for c in bc], dtype=np.int32)
    dof_a = np.array([c[1] for c in bc], dtype=np.int32)
    val_a = np.array([c[2] for c in bc], dtype=np.float64)
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    rc = gpu.monolis_b200_device_set_Dirichlet_bc_R(devm.p, d_b.data_ptr(), len(bc), node_a.ctypes.data_as(ip),
                                                     dof_a.ctypes.data_as(ip), val_a.ctypes.data_as(dp))
    assert rc == 0
    torch.cuda.synchronize()
    assert bits_equal(device_values(devm), host.values())
    assert bits_equal(d_b.cpu().numpy(), hb)


def test_device_assembled_solve_matches_host(gpu):
    """The C5 system assembled on the device solves to the same bits as the
    host-assembled one (same matrix, same kernels)."""
    import torch
    n = 10
    host = api.Monolis(gpu)
    bh, kappa, kref, elem = P.diffusion_kappa(host, n=n)
    devm = api.Monolis(gpu)
    devm.get_nonzero_pattern_flat(n ** 3, 8, 1, elem)
    assert gpu.monolis_b200_device_clear_matrix(devm.p) == 0
    d_elem, d_k, d_s = dev(elem), dev(kref.reshape(-1)), dev(kappa)
    assert gpu.monolis_b200_device_add_elements_R(devm.p, len(elem), 8, d_elem.data_ptr(), d_k.data_ptr(), 0,
                                                  d_s.data_ptr()) == 0
    d_b = dev(np.ones(n ** 3))
    nodes = np.arange(0, n ** 3, n, dtype=np.int32)
    zeros = np.zeros(len(nodes), dtype=np.int32)
    vals = np.zeros(len(nodes))
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    assert gpu.monolis_b200_device_set_Dirichlet_bc_R(devm.p, d_b.data_ptr(), len(nodes), nodes.ctypes.data_as(ip),
                                                      zeros.ctypes.data_as(ip), vals.ctypes.data_as(dp)) == 0
    torch.cuda.synchronize()
    assert bits_equal(device_values(devm), host.values())
    assert bits_equal(d_b.cpu().numpy(), bh)
    for m in (host, devm):
        m.quiet()
        m.set_method(api.ITER_CG)
        m.set_precond(api.PREC_DIAG)
        m.set_tolerance(1e-10)
    xh = np.zeros(n ** 3)
    host.solve(bh, xh)
    d_x = torch.zeros_like(d_b)
    assert devm.device_solve(d_b.data_ptr(), d_x.data_ptr()) == 0
    torch.cuda.synchronize()
    assert bits_equal(d_x.cpu().numpy(), xh)
    assert devm.get_converge_iter() == host.get_converge_iter()


def test_device_assembly_rejects_bad_input(gpu):
    n = 4
    elem = P.hex_elements(n)
    m = api.Monolis(gpu)
    m.get_nonzero_pattern_flat(n ** 3, 8, 1, elem)
    bad = elem.copy()
    bad[2, 3] = n ** 3 + 5
    d_elem, d_k = dev(bad), dev(np.eye(8).reshape(-1))
    assert gpu.monolis_b200_device_add_elements_R(m.p, len(bad), 8, d_elem.data_ptr(), d_k.data_ptr(), 0, None) == 5
    # an element whose node pair is not in the pattern: nodes 0 and 63 share no element
    far = np.array([[0, 63, 0, 0, 0, 0, 0, 0]], dtype=np.int32)
    d_far = dev(far)
    assert gpu.monolis_b200_device_add_elements_R(m.p, 1, 8, d_far.data_ptr(), d_k.data_ptr(), 0, None) == 5
