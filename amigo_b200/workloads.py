"""Seeded synthetic KKT systems with the shapes of the benchmark workloads.

Every generator returns a :class:`KKTSystem`: one symmetric CSR over all
variables (full pattern, 0-based, sorted columns, diagonal always present,
int32 indices, float64 values) plus the separate diagonal vector that Amigo
adds during the factorization (Sigma + perturbation on primal rows, -delta on
constraint rows), as in ``SparseLDL::factor(diag)`` (include/sparse_ldl.h:136)
and ``InertiaCorrector._compute_perturbation``
(amigo/algorithm/solvers/inertia_correction.py:280-294).

Random draws use ``numpy.random.default_rng(seed)`` in the documented order,
so the oracle and the GPU path always see the same numbers.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np

__all__ = [
    "KKTSystem",
    "csr_from_coo",
    "optimal_control_kkt",
    "plane_stress_kkt",
    "batched_optimal_control",
    "poisson_2d",
    "dense_to_csr",
]


@dataclasses.dataclass
class KKTSystem:
    n: int
    rowp: np.ndarray  # int32 [n+1]
    cols: np.ndarray  # int32 [nnz]
    vals: np.ndarray  # float64 [nnz]
    diag: np.ndarray  # float64 [n], added to the diagonal during factor
    rhs: np.ndarray  # float64 [n, nrhs], Fortran order
    n_primal: int
    n_con: int
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.rowp[-1])

    @property
    def expected_inertia(self) -> tuple[int, int]:
        return (self.n_primal, self.n_con)

    def to_dense(self) -> np.ndarray:
        """Dense K (+diag) for small systems."""
        a = np.zeros((self.n, self.n))
        r = np.repeat(np.arange(self.n), np.diff(self.rowp))
        np.add.at(a, (r, self.cols), self.vals)
        a[np.arange(self.n), np.arange(self.n)] += self.diag
        return a

    def matvec(self, x: np.ndarray) -> np.ndarray:
        """y = (K + diag) x in float64 for x of shape [n] or [n, k]."""
        r = np.repeat(np.arange(self.n), np.diff(self.rowp))
        x2 = x.reshape(self.n, -1)
        y = np.zeros_like(x2, dtype=np.float64)
        np.add.at(y, r, self.vals[:, None] * x2[self.cols])
        y += self.diag[:, None] * x2
        return y.reshape(x.shape)

    def inf_norm(self) -> float:
        """||K + diag||_inf."""
        r = np.repeat(np.arange(self.n), np.diff(self.rowp))
        a = np.abs(self.vals).copy()
        dpos = self.cols == r
        a[dpos] = np.abs(self.vals[dpos] + self.diag[r[dpos]])
        return float(np.max(np.bincount(r, weights=a, minlength=self.n)))


def csr_from_coo(n: int, rows, cols, vals, ensure_diagonal: bool = True):
    """Sum duplicates, sort columns and (optionally) insert explicit zeros on
    the diagonal so that every row holds its diagonal entry."""
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    vals = np.asarray(vals, dtype=np.float64)
    if ensure_diagonal:
        d = np.arange(n, dtype=np.int64)
        rows = np.concatenate([rows, d])
        cols = np.concatenate([cols, d])
        vals = np.concatenate([vals, np.zeros(n)])
    key = rows * n + cols
    order = np.argsort(key, kind="stable")
    key = key[order]
    vals = vals[order]
    uniq, start = np.unique(key, return_index=True)
    summed = np.add.reduceat(vals, start) if len(vals) else vals
    r = (uniq // n).astype(np.int64)
    c = (uniq % n).astype(np.int32)
    rowp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rowp, r + 1, 1)
    rowp = np.cumsum(rowp).astype(np.int32)
    return rowp, c, summed.astype(np.float64)


def dense_to_csr(a: np.ndarray, keep_zeros_on_diag: bool = True):
    """CSR of the nonzeros of a dense symmetric matrix (diagonal kept)."""
    n = a.shape[0]
    r, c = np.nonzero(a)
    return csr_from_coo(n, r, c, a[r, c], ensure_diagonal=keep_zeros_on_diag)


def _sym(rows, cols, vals):
    """Append the transpose of the off-diagonal entries."""
    rows = np.asarray(rows)
    cols = np.asarray(cols)
    vals = np.asarray(vals)
    off = rows != cols
    return (
        np.concatenate([rows, cols[off]]),
        np.concatenate([cols, rows[off]]),
        np.concatenate([vals, vals[off]]),
    )


def optimal_control_kkt(
    N: int = 1000,
    nx: int = 4,
    nu: int = 2,
    nrhs: int = 8,
    seed: int = 0,
    delta: float = 1e-8,
    rng: np.random.Generator | None = None,
    A_scale: np.ndarray | None = None,
) -> KKTSystem:
    """Discrete optimal-control KKT system (the N=1000, nx=4, nu=2 workload
    and the per-system generator of the batched and differentiation ones).

    Variable order: stage k primals ``[x_k (nx), u_k (nu)]`` at
    ``(nx+nu)*k``, then the multipliers of defect k (``x_{k+1} - A_k x_k -
    B_k u_k = 0``, k = 0..N-2) at ``(nx+nu)*N + nx*k``.

    Draw order from ``default_rng(seed)``: M (N, m, m) standard normal with
    m = nx+nu; A (N-1, nx, nx) = I + 0.1 N(0,1); B (N-1, nx, nu) N(0,1);
    log(Sigma) uniform on [ln 1e-6, ln 1e6] (N*m); RHS (n, nrhs) N(0,1).
    ``A_scale`` (N-1,) optionally multiplies each A_k (used for parameter
    sensitivities).
    """
    if rng is None:
        rng = np.random.default_rng(seed)
    m = nx + nu
    n_primal = N * m
    n_con = (N - 1) * nx
    n = n_primal + n_con

    M = rng.standard_normal((N, m, m))
    A = np.eye(nx)[None] + 0.1 * rng.standard_normal((N - 1, nx, nx))
    B = rng.standard_normal((N - 1, nx, nu))
    sigma = np.exp(rng.uniform(math.log(1e-6), math.log(1e6), size=n_primal))
    rhs = rng.standard_normal((n, nrhs))
    if A_scale is not None:
        A = A * np.asarray(A_scale, dtype=np.float64)[:, None, None]

    H = M @ M.transpose(0, 2, 1) / m + 1e-2 * np.eye(m)[None]
    base = (np.arange(N) * m)[:, None, None]
    hr = np.broadcast_to(base + np.arange(m)[None, :, None], H.shape)
    hc = np.broadcast_to(base + np.arange(m)[None, None, :], H.shape)
    rows = [hr.ravel()]
    cols = [hc.ravel()]
    vals = [H.ravel()]

    k = np.arange(N - 1)
    lam = n_primal + nx * k  # first multiplier row of defect k
    # +I on x_{k+1}
    li = (lam[:, None] + np.arange(nx)[None]).ravel()
    xi = ((k + 1)[:, None] * m + np.arange(nx)[None]).ravel()
    rows.append(li)
    cols.append(xi)
    vals.append(np.ones(li.shape))
    # -A_k on x_k
    ar = np.broadcast_to(lam[:, None, None] + np.arange(nx)[None, :, None], A.shape)
    ac = np.broadcast_to((k * m)[:, None, None] + np.arange(nx)[None, None, :], A.shape)
    rows.append(ar.ravel())
    cols.append(ac.ravel())
    vals.append(-A.ravel())
    # -B_k on u_k
    br = np.broadcast_to(lam[:, None, None] + np.arange(nx)[None, :, None], B.shape)
    bc = np.broadcast_to((k * m + nx)[:, None, None] + np.arange(nu)[None, None, :], B.shape)
    rows.append(br.ravel())
    cols.append(bc.ravel())
    vals.append(-B.ravel())

    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    # constraint blocks appear once (lower), mirror them
    is_con = r >= n_primal
    r2 = np.concatenate([r, c[is_con]])
    c2 = np.concatenate([c, r[is_con]])
    v2 = np.concatenate([v, v[is_con]])
    rowp, colsx, valsx = csr_from_coo(n, r2, c2, v2)

    diag = np.empty(n)
    diag[:n_primal] = sigma
    diag[n_primal:] = -delta
    return KKTSystem(
        n=n,
        rowp=rowp,
        cols=colsx,
        vals=valsx,
        diag=diag,
        rhs=np.asfortranarray(rhs),
        n_primal=n_primal,
        n_con=n_con,
        name=f"optimal_control_N{N}_nx{nx}_nu{nu}",
    )


def batched_optimal_control(
    num_systems: int = 512,
    nmin: int = 50,
    nmax: int = 400,
    nx: int = 6,
    nu: int = 3,
    seed: int = 0,
    nrhs: int = 1,
) -> list[KKTSystem]:
    """Many independent optimal-control systems of uneven size: N_i drawn
    uniformly from {nmin..nmax} first, then each system from the same
    generator stream in order."""
    rng = np.random.default_rng(seed)
    Ns = rng.integers(nmin, nmax + 1, size=num_systems)
    return [
        optimal_control_kkt(int(Ni), nx=nx, nu=nu, nrhs=nrhs, rng=rng) for Ni in Ns
    ]


def _q1_plane_stress_ke(nu: float = 0.3) -> np.ndarray:
    """8x8 stiffness of a unit-modulus square bilinear (Q1) element in plane
    stress, 2x2 Gauss quadrature. Node order (-1,-1), (1,-1), (1,1), (-1,1);
    dofs (x, y) per node. For a square element the 2D stiffness does not
    depend on its size."""
    D = (1.0 / (1.0 - nu * nu)) * np.array(
        [[1.0, nu, 0.0], [nu, 1.0, 0.0], [0.0, 0.0, (1.0 - nu) / 2.0]]
    )
    xi_n = np.array([-1.0, 1.0, 1.0, -1.0])
    eta_n = np.array([-1.0, -1.0, 1.0, 1.0])
    g = 1.0 / math.sqrt(3.0)
    ke = np.zeros((8, 8))
    for xi in (-g, g):
        for eta in (-g, g):
            dN_dxi = 0.25 * xi_n * (1 + eta * eta_n)
            dN_deta = 0.25 * eta_n * (1 + xi * xi_n)
            # unit-size element mapped from [-1,1]^2: J = h/2 I, so with
            # h = 2 the Jacobian is the identity and the result is exact for
            # every h (2D stiffness is size independent)
            Bm = np.zeros((3, 8))
            Bm[0, 0::2] = dN_dxi
            Bm[1, 1::2] = dN_deta
            Bm[2, 0::2] = dN_deta
            Bm[2, 1::2] = dN_dxi
            ke += Bm.T @ D @ Bm
    return ke


def plane_stress_kkt(
    nel: int = 256,
    seed: int = 0,
    nrhs_random: int = 4,
    delta: float = 1e-8,
    nu: float = 0.3,
) -> KKTSystem:
    """SAND-style PDE-constrained KKT system on an nel x nel Q1 plane-stress
    mesh (the 256 x 256 workload).

    Unknowns: u (2 (nel+1)^2 displacements), rho (nel^2 densities), lambda
    (2 (nel+1)^2 equilibrium multipliers), in that order. Blocks: lambda-u =
    K(rho) = sum_e rho_e^3 K_e; lambda-rho: dK(rho)u0/drho_e = 3 rho_e^2 K_e
    u0_e; rho-rho: 1e-3 I; u-u: 0. The left edge is clamped: a clamped dof d
    keeps only the (lambda_d, u_d) = 1 coupling and no K or G entries. Diagonal
    vector: 0 on u, Sigma log-uniform on [1e-4, 1e4] on rho, -delta on lambda.
    RHS: column 0 a unit load (-1 in y at the middle node of the right edge,
    in the lambda block), then ``nrhs_random`` N(0,1) columns.

    Draw order from ``default_rng(seed)``: rho U[0.3, 1] (nel^2), u0 N(0,1)
    (2 (nel+1)^2), log(Sigma) (nel^2), random RHS (n, nrhs_random).
    """
    rng = np.random.default_rng(seed)
    nn1 = nel + 1
    nnode = nn1 * nn1
    nu_dof = 2 * nnode
    ne = nel * nel
    off_rho = nu_dof
    off_lam = nu_dof + ne
    n = off_lam + nu_dof
    n_primal = nu_dof + ne

    rho = rng.uniform(0.3, 1.0, size=ne)
    u0 = rng.standard_normal(nu_dof)
    sigma = np.exp(rng.uniform(math.log(1e-4), math.log(1e4), size=ne))
    rhs_r = rng.standard_normal((n, nrhs_random))

    ke = _q1_plane_stress_ke(nu)
    ex, ey = np.meshgrid(np.arange(nel), np.arange(nel), indexing="xy")
    ex = ex.ravel()
    ey = ey.ravel()
    n0 = ex + ey * nn1
    nodes = np.stack([n0, n0 + 1, n0 + 1 + nn1, n0 + nn1], axis=1)  # (ne, 4)
    edofs = np.empty((ne, 8), dtype=np.int64)
    edofs[:, 0::2] = 2 * nodes
    edofs[:, 1::2] = 2 * nodes + 1

    clamped = np.zeros(nu_dof, dtype=bool)
    left = np.arange(nn1) * nn1  # nodes with x index 0
    clamped[2 * left] = True
    clamped[2 * left + 1] = True

    # lambda-u block: K(rho)
    kr = np.broadcast_to(edofs[:, :, None], (ne, 8, 8))
    kc = np.broadcast_to(edofs[:, None, :], (ne, 8, 8))
    kv = (rho**3)[:, None, None] * ke[None]
    keep = ~(clamped[kr] | clamped[kc])
    rows = [off_lam + kr[keep]]
    cols = [kc[keep]]
    vals = [kv[keep]]
    # lambda-rho block: G[:, e] = 3 rho_e^2 K_e u0_e
    ge = 3.0 * (rho**2)[:, None] * np.einsum("ab,eb->ea", ke, u0[edofs])
    gkeep = ~clamped[edofs]
    rows.append(off_lam + edofs[gkeep])
    cols.append(np.broadcast_to((off_rho + np.arange(ne))[:, None], (ne, 8))[gkeep])
    vals.append(ge[gkeep])
    # clamped dofs: identity coupling
    cd = np.nonzero(clamped)[0]
    rows.append(off_lam + cd)
    cols.append(cd)
    vals.append(np.ones(len(cd)))
    # rho-rho: 1e-3 I
    rr = off_rho + np.arange(ne)
    rows.append(rr)
    cols.append(rr)
    vals.append(np.full(ne, 1e-3))

    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    r2, c2, v2 = _sym(r, c, v)
    rowp, colsx, valsx = csr_from_coo(n, r2, c2, v2)

    diag = np.zeros(n)
    diag[off_rho:off_lam] = sigma
    diag[off_lam:] = -delta

    rhs = np.zeros((n, 1 + nrhs_random))
    load_node = nel + (nel // 2) * nn1  # right edge, middle
    rhs[off_lam + 2 * load_node + 1, 0] = -1.0
    rhs[:, 1:] = rhs_r
    return KKTSystem(
        n=n,
        rowp=rowp,
        cols=colsx,
        vals=valsx,
        diag=diag,
        rhs=np.asfortranarray(rhs),
        n_primal=n_primal,
        n_con=nu_dof,
        name=f"plane_stress_{nel}x{nel}",
    )


def _q1_hex_ke(nu: float = 0.3) -> np.ndarray:
    """24x24 stiffness of a unit-modulus, unit-cube trilinear (Q1) hex
    element, 2x2x2 Gauss quadrature. Node order: the bottom face (z = -1)
    (-1,-1), (1,-1), (1,1), (-1,1), then the top face (z = +1) in the same
    order; dofs (x, y, z) per node. Strains in Voigt order xx, yy, zz, xy,
    yz, zx."""
    lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = 1.0 / (2.0 * (1.0 + nu))
    D = np.zeros((6, 6))
    D[:3, :3] = lam
    D[np.arange(3), np.arange(3)] += 2.0 * mu
    D[np.arange(3, 6), np.arange(3, 6)] = mu
    xn = np.array([-1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0, -1.0])
    yn = np.array([-1.0, -1.0, 1.0, 1.0, -1.0, -1.0, 1.0, 1.0])
    zn = np.array([-1.0, -1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0])
    g = 1.0 / math.sqrt(3.0)
    ke = np.zeros((24, 24))
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                # reference-cube derivatives; the unit cube maps with
                # x = (xi + 1) / 2, so d/dx = 2 d/dxi and det J = 1/8
                dx = 2.0 * 0.125 * xn * (1 + eta * yn) * (1 + zeta * zn)
                dy = 2.0 * 0.125 * yn * (1 + xi * xn) * (1 + zeta * zn)
                dz = 2.0 * 0.125 * zn * (1 + xi * xn) * (1 + eta * yn)
                Bm = np.zeros((6, 24))
                Bm[0, 0::3] = dx
                Bm[1, 1::3] = dy
                Bm[2, 2::3] = dz
                Bm[3, 0::3] = dy
                Bm[3, 1::3] = dx
                Bm[4, 1::3] = dz
                Bm[4, 2::3] = dy
                Bm[5, 2::3] = dx
                Bm[5, 0::3] = dz
                ke += 0.125 * (Bm.T @ D @ Bm)
    return ke


def hex_elasticity_kkt(
    nel: int = 48,
    seed: int = 0,
    nrhs_random: int = 4,
    delta: float = 1e-8,
    nu: float = 0.3,
    sigma_range: tuple[float, float] = (1e-6, 1e6),
) -> KKTSystem:
    """The 3D counterpart of :func:`plane_stress_kkt` with a dense row (the
    48^3 hex workload): an nel^3 mesh of unit-cube Q1 hex elements.

    Unknowns, in order: u (3 (nel+1)^3 displacements), rho (nel^3
    densities), lambda (3 (nel+1)^3 equilibrium multipliers), mu (one volume
    multiplier). Blocks: lambda-u = K(rho) = sum_e rho_e^3 K_e; lambda-rho:
    3 rho_e^2 K_e u0_e; mu-rho: the element volumes (1 each), a dense row;
    rho-rho: 1e-3 I; u-u: 0. The face x = 0 is clamped: a clamped dof d
    keeps only the (lambda_d, u_d) = 1 coupling. Diagonal vector: 0 on u,
    Sigma log-uniform on ``sigma_range`` on rho, -delta on lambda and mu.
    Expected inertia: (number of u and rho, number of lambda and mu). RHS:
    column 0 a unit load (-1 in z at the centre node of the face x = nel, in
    the lambda block), then ``nrhs_random`` N(0,1) columns.

    Draw order from ``default_rng(seed)``: rho U[0.3, 1] (nel^3), u0 N(0,1)
    (3 (nel+1)^3), log(Sigma) (nel^3), random RHS (n, nrhs_random).
    """
    rng = np.random.default_rng(seed)
    nn1 = nel + 1
    nnode = nn1**3
    nu_dof = 3 * nnode
    ne = nel**3
    off_rho = nu_dof
    off_lam = nu_dof + ne
    off_mu = off_lam + nu_dof
    n = off_mu + 1
    n_primal = nu_dof + ne

    rho = rng.uniform(0.3, 1.0, size=ne)
    u0 = rng.standard_normal(nu_dof)
    sigma = np.exp(rng.uniform(math.log(sigma_range[0]), math.log(sigma_range[1]), size=ne))
    rhs_r = rng.standard_normal((n, nrhs_random))

    ke = _q1_hex_ke(nu)
    ex, ey, ez = np.meshgrid(np.arange(nel), np.arange(nel), np.arange(nel), indexing="ij")
    n0 = (ex + ey * nn1 + ez * nn1 * nn1).ravel()
    face = np.stack([n0, n0 + 1, n0 + 1 + nn1, n0 + nn1], axis=1)
    nodes = np.concatenate([face, face + nn1 * nn1], axis=1)  # (ne, 8)
    edofs = np.empty((ne, 24), dtype=np.int64)
    for d in range(3):
        edofs[:, d::3] = 3 * nodes + d

    clamped = np.zeros(nu_dof, dtype=bool)
    jj, kk = np.meshgrid(np.arange(nn1), np.arange(nn1), indexing="ij")
    x0 = (jj * nn1 + kk * nn1 * nn1).ravel()  # nodes with x index 0
    for d in range(3):
        clamped[3 * x0 + d] = True

    kr = np.broadcast_to(edofs[:, :, None], (ne, 24, 24))
    kc = np.broadcast_to(edofs[:, None, :], (ne, 24, 24))
    keep = ~(clamped[kr] | clamped[kc])
    kv = (rho**3)[:, None, None] * ke[None]
    rows = [off_lam + kr[keep]]
    cols = [kc[keep]]
    vals = [kv[keep]]
    ge = 3.0 * (rho**2)[:, None] * np.einsum("ab,eb->ea", ke, u0[edofs])
    gkeep = ~clamped[edofs]
    rows.append(off_lam + edofs[gkeep])
    cols.append(np.broadcast_to((off_rho + np.arange(ne))[:, None], (ne, 24))[gkeep])
    vals.append(ge[gkeep])
    cd = np.nonzero(clamped)[0]
    rows.append(off_lam + cd)
    cols.append(cd)
    vals.append(np.ones(len(cd)))
    rr = off_rho + np.arange(ne)
    rows.append(rr)
    cols.append(rr)
    vals.append(np.full(ne, 1e-3))
    # the volume constraint: sum_e rho_e (unit volumes)
    rows.append(np.full(ne, off_mu))
    cols.append(rr)
    vals.append(np.ones(ne))

    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    r2, c2, v2 = _sym(r, c, v)
    rowp, colsx, valsx = csr_from_coo(n, r2, c2, v2)

    diag = np.zeros(n)
    diag[off_rho:off_lam] = sigma
    diag[off_lam:] = -delta

    rhs = np.zeros((n, 1 + nrhs_random))
    mid = nel // 2
    load_node = nel + mid * nn1 + mid * nn1 * nn1  # face x = nel, centre
    rhs[off_lam + 3 * load_node + 2, 0] = -1.0
    rhs[:, 1:] = rhs_r
    return KKTSystem(
        n=n,
        rowp=rowp,
        cols=colsx,
        vals=valsx,
        diag=diag,
        rhs=np.asfortranarray(rhs),
        n_primal=n_primal,
        n_con=nu_dof + 1,
        name=f"hex_elasticity_{nel}^3",
    )


def poisson_2d(n: int, seed: int = 0):
    """5-point Laplacian on the (n-1)^2 interior grid of [0,1]^2, scaled by
    1/h^2, symmetrically permuted by ``np.random.permutation`` after
    ``np.random.seed(seed)`` (the reference's test matrix,
    tests/unit/test_ldl.py:85-118). Columns are sorted; the reference keeps
    scipy's row-slicing order, which does not change the factorization."""
    h = 1.0 / n
    m = n - 1
    state = np.random.get_state()
    np.random.seed(seed)
    perm = np.random.permutation(m * m)
    np.random.set_state(state)
    jj, ii = np.meshgrid(np.arange(m), np.arange(m), indexing="ij")
    jj = jj.ravel()
    ii = ii.ravel()
    me = jj * m + ii  # kron(I, T) + kron(T, I) numbering
    rows, cols, vals = [me], [me], [np.full(me.shape, 4.0 / h**2)]
    for dj, di in ((0, 1), (0, -1), (1, 0), (-1, 0)):
        ok = (ii + di >= 0) & (ii + di < m) & (jj + dj >= 0) & (jj + dj < m)
        rows.append(me[ok])
        cols.append((jj[ok] + dj) * m + ii[ok] + di)
        vals.append(np.full(int(ok.sum()), -1.0 / h**2))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    v = np.concatenate(vals)
    # permuted matrix P A P^T: new index of old row r is inv[r]
    inv = np.empty_like(perm)
    inv[perm] = np.arange(m * m)
    return csr_from_coo(m * m, inv[r], inv[c], v)
