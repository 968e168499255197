"""The multigrid hierarchy of the inner solve's preconditioner, built on the
host (csrc/host/amg.cpp through tg_amg_host_build) from a seeded 3D
finite-volume M-matrix, checked without a device:

- level 0 is the matrix given, and every restriction is the transpose of its
  prolongator;
- every coarse operator is the Galerkin product R A P with its weak entries
  (|g_ij| < 0.01 sqrt(g_ii g_jj)) lumped into the diagonal: kept entries are
  the product's, row sums are the product's, and the operator is symmetric;
- coarsening stops at 1,000 rows or fewer;
- the V(1,1)-cycle the device runs (damped Jacobi 0.9 on both sides, a dense
  solve on the coarsest level), restated here in numpy, preconditions CG to
  a relative residual of 1e-8 in a small fraction of the Jacobi-CG
  iterations, with the exact level-0 operator and with the one the device's
  smoothing pass applies (bf16 couplings, FP32 row sums);
- the same cycle on the inner system of a generated tip (an irregular
  Voronoi graph), assembled from the mesh arrays as the device assembles it."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from tapsim_modified_b200 import _native as N

DROP = 0.01       # AmgOptions::coarse_drop
SMOOTH = 0.9      # the device cycle's damped-Jacobi weight


def _poisson(m=32, seed=5):
    """7-point finite-volume operator on an m^3 grid: seeded couplings in
    [0.5, 2] and a Dirichlet coupling to the outside on boundary faces."""
    rng = np.random.default_rng(seed)
    n = m ** 3
    idx = np.arange(n).reshape(m, m, m)
    rows, cols, vals = [], [], []
    diag = np.zeros(n)
    for axis in range(3):
        a = np.moveaxis(idx, axis, 0)
        i, j = a[:-1].ravel(), a[1:].ravel()
        c = rng.uniform(0.5, 2.0, i.size)
        rows += [i, j]
        cols += [j, i]
        vals += [-c, -c]
        np.add.at(diag, i, c)
        np.add.at(diag, j, c)
        for face in (a[0].ravel(), a[-1].ravel()):
            np.add.at(diag, face, rng.uniform(0.5, 2.0, face.size))
    rows.append(np.arange(n))
    cols.append(np.arange(n))
    vals.append(diag)
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sort_indices()
    return A


def _matrix(h, level, which):
    rows, cols, nnz = C.c_int32(), C.c_int32(), C.c_int64()
    L = N.lib()
    assert L.tg_amg_host_matrix(h, level, which, C.byref(rows), C.byref(cols), C.byref(nnz), None, None, None) == 0
    ptr = np.empty(rows.value + 1, np.int32)
    col = np.empty(nnz.value, np.int32)
    val = np.empty(nnz.value, np.float64)
    assert L.tg_amg_host_matrix(h, level, which, C.byref(rows), C.byref(cols), C.byref(nnz), N.ptr(ptr), N.ptr(col),
                                N.ptr(val)) == 0
    return sp.csr_matrix((val, col, ptr), shape=(rows.value, cols.value))


@pytest.fixture(scope="module")
def hierarchy():
    A = _poisson()
    ptr, col, val = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    h = C.c_void_p()
    L = N.lib()
    assert L.tg_amg_host_build(A.shape[0], N.ptr(ptr), N.ptr(col), N.ptr(val), C.byref(h)) == 0
    levels = L.tg_amg_host_levels(h)
    As = [_matrix(h, l, 0) for l in range(levels)]
    Ps = [_matrix(h, l, 1) for l in range(levels - 1)]
    Rs = [_matrix(h, l, 2) for l in range(levels - 1)]
    with pytest.raises(AssertionError):
        _matrix(h, levels - 1, 1)  # the coarsest level has no prolongator
    L.tg_amg_host_destroy(h)
    return A, As, Ps, Rs


def test_levels_and_transfer_operators(hierarchy):
    A, As, Ps, Rs = hierarchy
    assert len(As) >= 3
    assert (As[0] != A).nnz == 0
    assert As[-1].shape[0] <= 1000
    for l, (P, R) in enumerate(zip(Ps, Rs)):
        assert P.shape == (As[l].shape[0], As[l + 1].shape[0])
        assert (R != P.T.tocsr()).nnz == 0, l


def test_coarse_operators_are_truncated_galerkin_products(hierarchy):
    _, As, Ps, Rs = hierarchy
    dropped = 0
    for l in range(len(Ps)):
        G = (Rs[l] @ As[l] @ Ps[l]).tocsr()
        Ac = As[l + 1].tocsr()
        scale = np.abs(G).max()
        assert abs(Ac - Ac.T).max() <= 1e-12 * scale, l
        g = G.diagonal()
        # kept off-diagonal entries are the product's
        coo = Ac.tocoo()
        off = coo.row != coo.col
        gk = np.asarray(G[coo.row[off], coo.col[off]]).ravel()
        assert np.abs(coo.data[off] - gk).max() <= 1e-12 * scale, l
        # the product's entries that are missing are the weak ones
        D = (G - Ac).tocoo()
        miss = (D.row != D.col) & (np.abs(D.data) > 1e-12 * scale)
        assert np.all(np.abs(D.data[miss]) < DROP * np.sqrt(g[D.row[miss]] * g[D.col[miss]])), l
        dropped += int(miss.sum())
        # lumping keeps every row sum
        rs_g = np.asarray(G.sum(axis=1)).ravel()
        rs_a = np.asarray(Ac.sum(axis=1)).ravel()
        assert np.abs(rs_a - rs_g).max() <= 1e-10 * np.abs(G).sum(axis=1).max(), l
    assert dropped > 0


def _pcg(A, b, prec, tol=1e-8, maxit=2000):
    x = np.zeros_like(b)
    r = b.copy()
    z = prec(r)
    p = z.copy()
    rz = r @ z
    b2 = b @ b
    for it in range(1, maxit + 1):
        q = A @ p
        alpha = rz / (p @ q)
        x += alpha * p
        r -= alpha * q
        if r @ r <= tol * tol * b2:
            return it, x
        z = prec(r)
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return maxit, x


def _bf16(x):
    """Round to the nearest bf16 (ties to even), returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _level0_bf16(A):
    """The operator the device's level-0 smoothing pass applies: FP32
    couplings rounded to bf16, and the diagonal g + sum of the rounded
    couplings, g being the FP32 operator's row sum."""
    A32 = A.astype(np.float32).tocsr()
    d = A32.diagonal().astype(np.float64)
    off = A32 - sp.diags(A32.diagonal())
    off.eliminate_zeros()
    a = -off.data                                    # couplings, positive
    g = d - np.asarray(sp.csr_matrix((a.astype(np.float64), off.indices, off.indptr), shape=A.shape).sum(axis=1)).ravel()
    ah = _bf16(a).astype(np.float64)
    Oh = sp.csr_matrix((ah, off.indices, off.indptr), shape=A.shape)
    return (sp.diags(g + np.asarray(Oh.sum(axis=1)).ravel()) - Oh).tocsr()


@pytest.mark.parametrize("level0", ["fp64", "bf16"])
def test_v_cycle_preconditions_cg(hierarchy, level0):
    A, As, Ps, Rs = hierarchy
    coarse_inv = np.linalg.inv(As[-1].toarray())
    diags = [M.diagonal() for M in As]
    ops = list(As)
    if level0 == "bf16":
        ops[0] = _level0_bf16(A)
        # symmetric, with the FP32 operator's row sums, and within 2^-8 of it
        # in every Rayleigh quotient
        assert abs(ops[0] - ops[0].T).max() == 0.0
        A32 = A.astype(np.float32).astype(np.float64)
        assert np.abs(np.asarray(ops[0].sum(axis=1)).ravel() - np.asarray(A32.sum(axis=1)).ravel()).max() <= \
            1e-6 * np.abs(A).sum(axis=1).max()
        v = np.random.default_rng(3).standard_normal((A.shape[0], 8))
        q = np.einsum("ij,ij->j", v, ops[0] @ v) / np.einsum("ij,ij->j", v, A @ v)
        assert np.all(np.abs(q - 1.0) <= 2.0 ** -8), q

    def cycle(l, b):
        if l == len(As) - 1:
            return coarse_inv @ b
        y = SMOOTH * b / diags[l]
        t = b - ops[l] @ y
        y = y + Ps[l] @ cycle(l + 1, Rs[l] @ t)
        return y + SMOOTH * (b - ops[l] @ y) / diags[l]

    b = np.random.default_rng(11).standard_normal(A.shape[0])
    it_mg, x = _pcg(A, b, lambda r: cycle(0, r))
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
    d = A.diagonal()
    it_j, _ = _pcg(A, b, lambda r: r / d)
    print("CG iterations to 1e-8 with the", level0, "level-0 operator: multigrid", it_mg, "Jacobi", it_j)
    assert it_mg <= 25
    assert it_mg <= 0.25 * it_j


def test_bad_input_is_rejected():
    L = N.lib()
    h = C.c_void_p()
    ptr = np.array([0, 1, 2], np.int32)
    col = np.array([0, 5], np.int32)  # column out of range
    val = np.array([1.0, 1.0])
    assert L.tg_amg_host_build(2, N.ptr(ptr), N.ptr(col), N.ptr(val), C.byref(h)) == N.TG_ERR_ARGUMENT
    assert not h.value
    assert L.tg_amg_host_levels(None) == 0


def _tip_v_system():
    """The inner system of a generated tip, as the device assembles it: rows
    of the free non-Neumann cells, off-diagonals -c_ij to free non-Neumann
    neighbours, and the diagonal sum c_ij over all non-Neumann neighbours
    (Dirichlet ones included)."""
    from conftest import SMALL_TIP
    from tapsim_modified_b200.tapsim import Mesh
    m = Mesh.from_tip(**dict(SMALL_TIP, cap_radius=4e-9, shank_length=6e-9, fine_shell=2e-9))
    a = m.arrays()
    n = m.num_nodes
    dirichlet = np.array([a["types"][int(t)]["dirichlet"] for t in a["type"]], bool)
    neumann = np.array([a["types"][int(t)]["neumann"] for t in a["type"]], bool)
    rp, col, c = a["row_ptr"], a["col"], a["coupling"]
    row = np.repeat(np.arange(n), np.diff(rp))
    live = ~neumann[col]
    diag = np.bincount(row[live], weights=c[live], minlength=n)
    free = ~dirichlet & ~neumann
    slot = np.full(n, -1)
    slot[free] = np.arange(free.sum())
    e = free[row] & free[col]
    nv = int(free.sum())
    A = sp.csr_matrix((np.concatenate([-c[e], diag[free]]),
                       (np.concatenate([slot[row[e]], np.arange(nv)]), np.concatenate([slot[col[e]], np.arange(nv)]))),
                      shape=(nv, nv))
    A.sort_indices()
    return A


def test_tip_v_system_hierarchy_preconditions_cg():
    """The same checks on the operator class the device solves: the V system
    of a 116k-cell generated tip (irregular Voronoi graph, graded cells)."""
    A = _tip_v_system()
    assert abs(A - A.T).max() <= 1e-12 * abs(A).max()
    ptr, col, val = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    h = C.c_void_p()
    L = N.lib()
    assert L.tg_amg_host_build(A.shape[0], N.ptr(ptr), N.ptr(col), N.ptr(val), C.byref(h)) == 0
    levels = L.tg_amg_host_levels(h)
    As = [_matrix(h, l, 0) for l in range(levels)]
    Ps = [_matrix(h, l, 1) for l in range(levels - 1)]
    L.tg_amg_host_destroy(h)
    assert levels >= 3 and As[-1].shape[0] <= 1000
    coarse_inv = np.linalg.inv(As[-1].toarray())
    diags = [M.diagonal() for M in As]
    ops = [_level0_bf16(A)] + As[1:]

    def cycle(l, b):
        if l == len(As) - 1:
            return coarse_inv @ b
        y = SMOOTH * b / diags[l]
        t = b - ops[l] @ y
        y = y + Ps[l] @ cycle(l + 1, Ps[l].T @ t)
        return y + SMOOTH * (b - ops[l] @ y) / diags[l]

    b = np.random.default_rng(13).standard_normal(A.shape[0])
    it_mg, x = _pcg(A, b, lambda r: cycle(0, r))
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
    d = A.diagonal()
    it_j, _ = _pcg(A, b, lambda r: r / d)
    print("tip V system", A.shape[0], "rows,", levels, "levels; CG iterations to 1e-8: multigrid", it_mg,
          "Jacobi", it_j)
    assert it_mg <= 30
    assert it_mg <= 0.2 * it_j


def _build(A):
    A = sp.csr_matrix(A)
    A.sort_indices()
    ptr, col, val = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    h = C.c_void_p()
    rc = N.lib().tg_amg_host_build(A.shape[0], N.ptr(ptr), N.ptr(col), N.ptr(val), C.byref(h))
    return rc, h


def test_small_matrix_is_one_level():
    """At most 1,000 rows: no coarsening, the matrix itself is the coarsest
    level (inverted densely on the device), with no transfer operators."""
    A = _poisson(m=8)  # 512 rows
    rc, h = _build(A)
    assert rc == 0
    L = N.lib()
    assert L.tg_amg_host_levels(h) == 1
    assert (_matrix(h, 0, 0) != A).nnz == 0
    rows = C.c_int32()
    assert L.tg_amg_host_matrix(h, 0, 1, C.byref(rows), None, None, None, None, None) == N.TG_ERR_ARGUMENT
    L.tg_amg_host_destroy(h)


def test_rows_without_neighbours_and_disconnected_blocks():
    """Rows without off-diagonal entries (cells whose neighbours are all
    Dirichlet) stay out of the coarse levels, and two disconnected blocks are
    coarsened apart: the prolongator has no entry that couples them, and the
    hierarchy still preconditions CG."""
    B = _poisson(m=14, seed=9)                       # 2,744 rows
    iso = sp.diags(np.full(300, 3.0))                # isolated rows
    A = sp.block_diag([B, iso, _poisson(m=14, seed=21)]).tocsr()
    rc, h = _build(A)
    assert rc == 0
    L = N.lib()
    levels = L.tg_amg_host_levels(h)
    assert levels >= 2
    As = [_matrix(h, l, 0) for l in range(levels)]
    Ps = [_matrix(h, l, 1) for l in range(levels - 1)]
    L.tg_amg_host_destroy(h)
    nb = B.shape[0]
    P = Ps[0].tocoo()
    assert not np.any((P.row >= nb) & (P.row < nb + 300)), "isolated rows enter the coarse space"
    first = set(P.col[P.row < nb].tolist())
    second = set(P.col[P.row >= nb + 300].tolist())
    assert first and second and not (first & second)
    coarse_inv = np.linalg.inv(As[-1].toarray())
    diags = [M.diagonal() for M in As]

    def cycle(l, b):
        if l == len(As) - 1:
            return coarse_inv @ b
        y = SMOOTH * b / diags[l]
        t = b - As[l] @ y
        y = y + Ps[l] @ cycle(l + 1, Ps[l].T @ t)
        return y + SMOOTH * (b - As[l] @ y) / diags[l]

    b = np.random.default_rng(2).standard_normal(A.shape[0])
    it, x = _pcg(A, b, lambda r: cycle(0, r))
    assert np.linalg.norm(b - A @ x) <= 1e-8 * np.linalg.norm(b)
    assert it <= 25


def test_non_positive_diagonal_is_a_host_error():
    A = _poisson(m=12).tolil()
    A[5, 5] = -1.0
    rc, h = _build(A)
    assert rc == N.TG_ERR_HOST
    assert not h.value


def test_worker_allocation_failure_is_an_error():
    """An allocation failure inside one of the build's worker threads comes
    back from the C ABI as TG_ERR_HOST with its message, instead of ending
    the process through std::terminate; every thread is joined, and the next
    build (hook off) succeeds.  Run in a child process, so that a regression
    (terminate) fails this test instead of ending the test session."""
    import subprocess
    import sys
    import textwrap
    from pathlib import Path
    code = textwrap.dedent("""
        import ctypes as C, sys
        import numpy as np
        sys.path.insert(0, %r)
        sys.path.insert(0, %r)
        import test_amg_host as T
        from tapsim_modified_b200 import _native as N
        L = N.lib()
        A = T._poisson(m=14, seed=3)                 # 2,744 rows: threaded passes
        L.tg_amg_host_inject_worker_failure(1)
        rc, h = T._build(A)
        msg = L.tg_last_error(None).decode()
        L.tg_amg_host_inject_worker_failure(0)
        assert rc == N.TG_ERR_HOST and not h.value, (rc, h.value)
        assert "bad_alloc" in msg or "alloc" in msg, msg
        rc, h = T._build(A)
        assert rc == 0 and L.tg_amg_host_levels(h) >= 2
        L.tg_amg_host_destroy(h)
        print("ok")
    """) % (str(Path(__file__).resolve().parent.parent), str(Path(__file__).resolve().parent))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
