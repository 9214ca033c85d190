"""Seeded synthetic problems for the benchmark configurations.

Each builder takes a `Monolis` (bound to any library exporting the monolis C
API) and assembles the system through that library's own pattern / assembly
/ Dirichlet calls, so the product and the oracle receive identical inputs.

Configurations (sizes are parameters; the defaults are the benchmark sizes):
  laplacian(n=32)         3D 7-point Laplacian, n^3 unknowns, ndof 1, diagonal 6,
                          -1 per grid edge, zero Dirichlet outside the grid,
                          b ~ U(0,1) (SplitMix64 seed 1); CG + DIAG.
  elasticity(n=128)       3D linear elasticity, n^3 nodes, (n-1)^3 trilinear hex8
                          elements, E = 1, nu = 0.3, 2x2x2 Gauss; face x = 0
                          clamped; body force (0, 0, -1) per unit volume plus an
                          N(0, 0.01) perturbation of the force density per dof
                          (seed 2); ndof 3; CG + DIAG (3x3 block Jacobi).
  convection_diffusion(n=256, peclet)
                          7-point first-order upwind, D = 1, velocity along
                          (1, 0.5, 0.25) scaled to cell Peclet |v|h/(2D), zero
                          Dirichlet outside, b ~ U(0,1) (seed 3); BiCGSTAB + DIAG.
  diffusion_kappa(n=128)  Q1 hex8 scalar diffusion, A = sum_e kappa_e K_e,
                          kappa_e ~ LogNormal(0, 1) (seed 5), zero Dirichlet on
                          x = 0, b = 1; the adjoint configuration.
Random numbers: SplitMix64 (Steele, Lea, Flood 2014) counter stream per seed,
53-bit uniforms; normals by Box-Muller.
"""
from __future__ import annotations

import numpy as np

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int, offset: int = 0) -> np.ndarray:
    """n outputs of the SplitMix64 generator started at `seed`, as uint64."""
    with np.errstate(over="ignore"):
        k = np.arange(offset + 1, offset + n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int, offset: int = 0) -> np.ndarray:
    return (splitmix64(seed, n, offset) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int, mu: float = 0.0, sigma: float = 1.0) -> np.ndarray:
    m = (n + 1) // 2
    u1 = uniform(seed, m, 0)
    u2 = uniform(seed, m, m)
    u1 = np.where(u1 <= 0.0, 1e-300, u1)
    rad = np.sqrt(-2.0 * np.log(u1))
    z = np.concatenate([rad * np.cos(2 * np.pi * u2), rad * np.sin(2 * np.pi * u2)])[:n]
    return mu + sigma * z


# ---------------------------------------------------------------------------
# Meshes (node id = ix + n*iy + n*n*iz)
# ---------------------------------------------------------------------------
def grid_edges(n: int):
    """2-node edges of an n^3 grid in the order of sample/cg_diag_3d/main.f90:
    node by node (x fastest), and per node its +x, +y, +z edge. Returns
    (edges[int32 E x 2], direction[int8 E])."""
    ids = np.arange(n ** 3, dtype=np.int64)
    ix, iy, iz = ids % n, (ids // n) % n, ids // (n * n)
    parts, dirs, keys = [], [], []
    for d, (ok, step) in enumerate([(ix < n - 1, 1), (iy < n - 1, n), (iz < n - 1, n * n)]):
        a = ids[ok]
        parts.append(np.stack([a, a + step], axis=1))
        dirs.append(np.full(len(a), d, dtype=np.int8))
        keys.append(a * 3 + d)
    e = np.concatenate(parts)
    d = np.concatenate(dirs)
    order = np.argsort(np.concatenate(keys), kind="stable")
    return e[order].astype(np.int32), d[order]


def hex_elements(n: int) -> np.ndarray:
    """(n-1)^3 trilinear hexahedra of an n^3 node grid, int32 (E x 8), element
    order x fastest, local nodes (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),..."""
    m = n - 1
    e = np.arange(m ** 3, dtype=np.int64)
    ex, ey, ez = e % m, (e // m) % m, e // (m * m)
    base = ex + n * ey + n * n * ez
    off = np.array([0, 1, 1 + n, n, n * n, 1 + n * n, 1 + n + n * n, n + n * n], dtype=np.int64)
    return (base[:, None] + off[None, :]).astype(np.int32)


_HEX_NAT = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def _hex_grads(h: float):
    """Shape-function gradients (8 x 3) at the 2x2x2 Gauss points of a cube of side h."""
    g = 1.0 / np.sqrt(3.0)
    out = []
    for gz in (-g, g):
        for gy in (-g, g):
            for gx in (-g, g):
                xi = np.array([gx, gy, gz])
                dN = np.empty((8, 3))
                for a in range(8):
                    s = _HEX_NAT[a]
                    f = 1.0 + s * xi
                    dN[a, 0] = s[0] * f[1] * f[2] / 8.0
                    dN[a, 1] = s[1] * f[0] * f[2] / 8.0
                    dN[a, 2] = s[2] * f[0] * f[1] / 8.0
                out.append(dN * (2.0 / h))  # dxi/dx = 2/h
    det_j = (h / 2.0) ** 3
    return out, det_j


def hex8_elasticity_ke(h: float, E: float = 1.0, nu: float = 0.3) -> np.ndarray:
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2 * mu
    D[3, 3] = D[4, 4] = D[5, 5] = mu
    grads, det_j = _hex_grads(h)
    K = np.zeros((24, 24))
    for dN in grads:
        Bm = np.zeros((6, 24))
        for a in range(8):
            dx, dy, dz = dN[a]
            c = 3 * a
            Bm[0, c] = dx
            Bm[1, c + 1] = dy
            Bm[2, c + 2] = dz
            Bm[3, c] = dy
            Bm[3, c + 1] = dx
            Bm[4, c + 1] = dz
            Bm[4, c + 2] = dy
            Bm[5, c] = dz
            Bm[5, c + 2] = dx
        K += Bm.T @ D @ Bm * det_j
    return K


def hex8_diffusion_ke(h: float) -> np.ndarray:
    grads, det_j = _hex_grads(h)
    K = np.zeros((8, 8))
    for dN in grads:
        K += dN @ dN.T * det_j
    return K


# ---------------------------------------------------------------------------
# Builders
# ---------------------------------------------------------------------------
def laplacian(m, n: int = 32, seed: int = 1, diag: float = 6.0):
    """C1. Returns b."""
    edges, _ = grid_edges(n)
    nn = n ** 3
    m.get_nonzero_pattern_flat(nn, 2, 1, edges)
    m.add_elements(np.arange(nn, dtype=np.int32), 1, np.array([diag]), 0)
    m.add_elements(edges, 2, np.array([0.0, -1.0, -1.0, 0.0]), 0)
    return uniform(seed, nn)


def convection_diffusion(m, n: int = 256, peclet: float = 0.5, seed: int = 3, D: float = 1.0):
    """C3 (system scaled by h^2). Returns b."""
    edges, d = grid_edges(n)
    nn = n ** 3
    vdir = np.array([1.0, 0.5, 0.25])
    hv = 2.0 * peclet * D * vdir  # h * v_d with |v|_inf h / (2D) = peclet
    m.get_nonzero_pattern_flat(nn, 2, 1, edges)
    m.add_elements(np.arange(nn, dtype=np.int32), 1, np.array([6.0 * D + hv.sum()]), 0)
    # edge (a, b = a + e_d): row a gets -D (downstream neighbour), row b gets
    # -D - h v_d (upstream neighbour, first-order upwind)
    val = np.zeros((len(edges), 4))
    val[:, 1] = -D
    val[:, 2] = -D - hv[d]
    m.add_elements(edges, 2, val.reshape(-1), 4)
    return uniform(seed, nn)


def _clamp_face_x0(m, n: int, ndof: int, b: np.ndarray):
    for node in range(0, n ** 3, n):  # ix == 0
        for k in range(ndof):
            m.set_Dirichlet_bc(b, node, k, 0.0)


def elasticity(m, n: int = 128, seed: int = 2, E: float = 1.0, nu: float = 0.3):
    """C2. Returns b (after the Dirichlet conditions)."""
    h = 1.0 / (n - 1)
    elem = hex_elements(n)
    nn = n ** 3
    m.get_nonzero_pattern_flat(nn, 8, 3, elem)
    m.add_elements(elem, 8, hex8_elasticity_ke(h, E, nu).reshape(-1), 0)
    # consistent nodal load of a constant force density: h^3/8 per node per element
    cnt = np.bincount(elem.reshape(-1), minlength=nn).astype(np.float64) * (h ** 3 / 8.0)
    f = np.zeros((nn, 3))
    f[:, 2] = -1.0
    f += normal(seed, nn * 3, 0.0, 0.01).reshape(nn, 3)
    b = np.ascontiguousarray((f * cnt[:, None]).reshape(-1))
    _clamp_face_x0(m, n, 3, b)
    return b


def diffusion_kappa(m, n: int = 128, seed: int = 5, kappa=None):
    """C5 forward system. Returns (b, kappa, K_ref, elem)."""
    h = 1.0 / (n - 1)
    elem = hex_elements(n)
    nn = n ** 3
    if kappa is None:
        kappa = np.exp(normal(seed, len(elem), 0.0, 1.0))
    kref = hex8_diffusion_ke(h)
    m.get_nonzero_pattern_flat(nn, 8, 1, elem)
    m.add_elements(elem, 8, kref.reshape(-1), 0, scale=kappa)
    b = np.ones(nn)
    _clamp_face_x0(m, n, 1, b)
    return b, kappa, kref, elem


def face_x0_fixed(n: int, ndof: int) -> np.ndarray:
    """Per-dof mask (int32, n^3 * ndof) of the dofs clamped on the x = 0 face."""
    fixed = np.zeros((n ** 3, ndof), dtype=np.int32)
    fixed[0::n, :] = 1
    return fixed.reshape(-1)


def smooth_target(n: int, seed: int = 5) -> np.ndarray:
    """x_target of the adjoint workload on the n^3 node grid of the unit cube:
    sin(pi x) sin(pi y) sin(pi z) plus 0.1 times a seeded smooth field (eight
    low-frequency sine modes with N(0,1) amplitudes)."""
    t = np.linspace(0.0, 1.0, n)
    z, y, x = np.meshgrid(t, t, t, indexing="ij")  # node id = ix + n*iy + n*n*iz
    field = np.zeros_like(x)
    amp = normal(seed + 1000, 8)
    modes = [(1, 2, 1), (2, 1, 1), (1, 1, 2), (2, 2, 1), (1, 2, 2), (2, 1, 2), (3, 1, 1), (1, 3, 2)]
    for a, (kx, ky, kz) in zip(amp, modes):
        field += a * np.sin(kx * np.pi * x) * np.sin(ky * np.pi * y) * np.sin(kz * np.pi * z)
    out = np.sin(np.pi * x) * np.sin(np.pi * y) * np.sin(np.pi * z) + 0.1 * field
    return np.ascontiguousarray(out.reshape(-1))


def fv_diffusion_csr(side: int, seed: int):
    """Cell-centred finite-volume diffusion on a side^3 cube of unit cells
    (7-point stencil): per-cell conductivity kappa ~ LogNormal(0, 1), face
    transmissibility the harmonic mean 2 k_i k_j / (k_i + k_j), zero Dirichlet
    outside (boundary face 2 k_i). Returns the block CSR (0-based offsets and
    columns, ascending columns, ndof 1): (index, item, val, kappa)."""
    n = side ** 3
    kappa = np.exp(normal(seed, n, 0.0, 1.0))
    c = np.arange(n, dtype=np.int64)
    ix, iy, iz = c % side, (c // side) % side, c // (side * side)
    offs = [-side * side, -side, -1, 0, 1, side, side * side]
    coord = [iz, iy, ix, None, ix, iy, iz]
    cols = np.full((n, 7), -1, dtype=np.int64)
    vals = np.zeros((n, 7))
    diag = np.zeros(n)
    for k, (o, q) in enumerate(zip(offs, coord)):
        if o == 0:
            continue
        ok = (q > 0) if o < 0 else (q < side - 1)
        j = c + o
        t = np.zeros(n)
        kj = kappa[np.where(ok, j, c)]
        t_int = 2.0 * kappa * kj / (kappa + kj)
        t = np.where(ok, t_int, 2.0 * kappa)
        diag += t
        cols[ok, k] = j[ok]
        vals[ok, k] = -t_int[ok]
    cols[:, 3] = c
    vals[:, 3] = diag
    valid = cols >= 0
    index = np.zeros(n + 1, dtype=np.int32)
    index[1:] = np.cumsum(valid.sum(axis=1))
    return index, cols[valid].astype(np.int32), np.ascontiguousarray(vals[valid]), kappa


def batch_sides(count: int = 512, seed: int = 4, lo: float = 10.0, hi: float = 60.0) -> np.ndarray:
    """Side lengths round(exp(U(ln lo, ln hi))) of the batched workload."""
    u = uniform(seed, count)
    return np.rint(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)


def csr_matvec(index, item, val, x):
    """y = A x for a 0-based scalar CSR (numpy, FP64)."""
    rows = np.repeat(np.arange(len(index) - 1), np.diff(index))
    return np.bincount(rows, weights=val * x[item], minlength=len(index) - 1)


def spmv_bytes(nz: int, n: int, ndof: int, value_bytes: int) -> int:
    """Algorithmic bytes of one block SpMV: every value and column id read
    once, the row offsets once, x read once and y written once."""
    return nz * (ndof * ndof * value_bytes + 4) + (n + 1) * 4 + 2 * n * ndof * value_bytes
