"""Known-answer tests of the oracle from the reference's mathematics (no GPU).

SH orthonormality (the check in GPU package/src/dist.cu:545-672), the exact radiological path in a
uniform medium and against an independent crossing-sort computation, the collimated source closed
form (JOSAA GPU Eq. 23, dist.cu:66-101), g = 0 keeps only l = 0 after scatter (prop_scat_dev),
linearity, the Neumann series against a dense direct solve of (I - DA) x = xi on a tiny grid, and
photon conservation without absorption (ComputePhotonNumber).
"""
import numpy as np
import pytest

from conftest import rel


def test_sh_orthonormal(oracle):
    L = 5
    C = (L + 1) ** 2
    x, w = np.polynomial.legendre.leggauss(24)  # exact for the product of two degree-5 polynomials
    nphi = 24
    G = np.zeros((C, C), np.complex128)
    for xi, wi in zip(x, w):
        th = np.arccos(xi)
        for k in range(nphi):
            Y = oracle.sh_complex(L, th, 2 * np.pi * k / nphi)
            G += wi * (2 * np.pi / nphi) * np.outer(np.conj(Y), Y)
    assert np.abs(G - np.eye(C)).max() < 1e-13


def test_sh_negative_m_symmetry(oracle):
    L = 4
    Y = oracle.sh_complex(L, 0.7, 2.1)
    for l in range(L + 1):
        for m in range(1, l + 1):
            assert abs(Y[l * l + l - m] - (-1) ** m * np.conj(Y[l * l + l + m])) < 1e-14


def _independent_path(mut, nx, ny, a, b, dx):
    """sum mu(v) * length(v) from crossing parameters sorted explicitly (no Siddon stepping)."""
    a = np.array(a, float)
    b = np.array(b, float)
    d = b - a
    alphas = [0.0, 1.0]
    for ax in range(3):
        if d[ax] != 0:
            for n in range(int(abs(d[ax]))):
                alphas.append((n + 0.5) / abs(d[ax]))
    alphas = np.unique(np.array(alphas))
    r = np.linalg.norm(d * dx)
    tot = 0.0
    for lo, hi in zip(alphas[:-1], alphas[1:]):
        mid = a + d * (lo + hi) / 2
        i, j, k = (int(np.floor(v + 0.5)) for v in mid)
        tot += mut[(i * ny + j) * nx + k] * (hi - lo) * r
    return tot


def test_path_integral(oracle):
    rng = np.random.default_rng(0)
    nx = ny = nz = 9
    dx = 0.1
    p = oracle.params(nx, ny, nz, dx, dx, dx, 1, 0.8, 1.0, 10.0)
    mut_u = np.full(nx * ny * nz, 1.3)
    mut = rng.uniform(0.1, 3.0, nx * ny * nz)
    for _ in range(60):
        a = rng.integers(0, 9, 3)
        b = rng.integers(0, 9, 3)
        if (a == b).all():
            continue
        r = np.linalg.norm((a - b) * dx)
        assert abs(oracle.path_integral(p, mut_u, a, b) - 1.3 * r) < 1e-13
        assert abs(oracle.path_integral(p, mut_u, a, b, fp32ref=True) - 1.3 * r) < 1e-6 * r
        exact = _independent_path(mut, nx, ny, a, b, dx)
        assert abs(oracle.path_integral(p, mut, a, b) - exact) < 1e-12 * max(exact, 1)
        assert abs(oracle.path_integral(p, mut, b, a) - exact) < 1e-12 * max(exact, 1)


def test_source_closed_form(oracle):
    rng = np.random.default_rng(1)
    n, L, dx = 6, 3, 0.1
    N = n ** 3
    mua = rng.uniform(0.01, 0.1, N)
    mus = rng.uniform(0.5, 2.0, N)
    g = 0.7
    p = oracle.params(n, n, n, dx, dx, dx, L, g, 1.0, 10.0)
    W = oracle.source(p, mua, mus, pos_x=0.01, pos_y=-0.01, mag=2.0, kind=oracle.SRC_COLUMN)
    cx = int(np.floor((0.01 + n * dx / 2) / dx))
    cy = int(np.floor((-0.01 + n * dx / 2) / dx))
    ref = np.zeros_like(W)
    att = 1.0
    for i in range(n):
        r = (i * n + cy) * n + cx
        mt = mua[r] + mus[r]
        for l in range(L + 1):
            ref[r, l * l + l] = 2.0 * g ** l * mus[r] / mt * np.sqrt((2 * l + 1) / (4 * np.pi)) * att * (
                1 - np.exp(-mt * dx)) / dx ** 3
        att *= np.exp(-mt * dx)
    assert rel(W, ref) < 1e-14


def test_isotropic_scatter_keeps_l0(oracle):
    rng = np.random.default_rng(2)
    n, L = 5, 2
    N, C = n ** 3, (L + 1) ** 2
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.0, 1.0, 10.0)
    W = rng.standard_normal((N, C)) + 0j
    out = oracle.apply(p, np.full(N, 0.02), np.full(N, 1.1), W, 1, 1)
    assert np.abs(out[:, 1:]).max() == 0.0
    assert np.abs(out[:, 0]).max() > 0


def test_linearity(oracle):
    rng = np.random.default_rng(3)
    n, L = 5, 2
    N, C = n ** 3, (L + 1) ** 2
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.8, 1.0, 10.0)
    mua, mus = rng.uniform(0.01, 0.1, N), rng.uniform(0.5, 2, N)
    W1 = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
    W2 = rng.standard_normal((N, C)) + 1j * rng.standard_normal((N, C))
    a, b = 0.3 - 1.2j, 2.5
    lhs = oracle.apply(p, mua, mus, a * W1 + b * W2)
    rhs = a * oracle.apply(p, mua, mus, W1) + b * oracle.apply(p, mua, mus, W2)
    assert rel(lhs, rhs) < 1e-14


def test_exact_and_cpu_models_share_the_operator(oracle):
    """In a uniform medium the exact path integral is mu_t r, so the exact model's operator equals
    the CPU package's (exact SH, exp(-mu_t r), 200x200 self term with per-axis half widths)."""
    rng = np.random.default_rng(4)
    n, L = 5, 3
    N, C = n ** 3, (L + 1) ** 2
    W = rng.standard_normal((N, C)) + 0j
    mua, mus = np.full(N, 0.02), np.full(N, 1.3)
    pe = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.8, 1.0, 10.0, mode=oracle.MODE_EXACT)
    pc = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.8, 1.0, 10.0, mode=oracle.MODE_CPU)
    assert rel(oracle.apply(pe, mua, mus, W), oracle.apply(pc, mua, mus, W)) < 1e-13


def test_neumann_equals_direct_solve(oracle):
    """sum_k (DA)^k xi == (I - DA)^-1 xi (dense LU) on a 3^3 grid, L = 1."""
    rng = np.random.default_rng(5)
    n, L = 3, 1
    N, C = n ** 3, (L + 1) ** 2
    mua, mus = rng.uniform(0.05, 0.2, N), rng.uniform(0.5, 1.5, N)
    p = oracle.params(n, n, n, 0.3, 0.3, 0.3, L, 0.6, 1.0, 10.0)
    M = np.zeros((N * C, N * C), np.complex128)
    for q in range(N * C):
        e = np.zeros(N * C, np.complex128)
        e[q] = 1.0
        M[:, q] = oracle.apply(p, mua, mus, e.reshape(N, C), 1, 1).ravel()
    assert np.abs(np.linalg.eigvals(M)).max() < 0.9
    xi = oracle.source(p, mua, mus, kind=oracle.SRC_COLUMN)
    x = np.linalg.solve(np.eye(N * C) - M, xi.ravel()).reshape(N, C)
    out, _, nt = oracle.neumann(p, mua, mus, xi, xi, 1, oracle.STOP_FIXED, max_terms=300)
    A_x = oracle.apply(p, mua, mus, x, 1, 0)
    assert rel(out, A_x) < 1e-12


def test_ballistic_only_image(oracle):
    n, L = 5, 2
    N, C = n ** 3, (L + 1) ** 2
    rng = np.random.default_rng(6)
    mua, mus = rng.uniform(0.01, 0.1, N), rng.uniform(0.5, 2, N)
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.8, 1.0, 10.0)
    tr, rf = oracle.images(p, mua, mus, np.zeros((N, C)), 0, mag=3.0)
    c = n // 2
    col = [(i * n + c) * n + c for i in range(n)]
    assert abs(tr[c, c] - 3.0 * np.exp(-np.sum((mua + mus)[col]) * 0.1)) < 1e-15
    tr[c, c] = 0
    assert np.abs(tr).max() == 0 and np.abs(rf).max() == 0


@pytest.mark.parametrize("l", range(6))
def test_exitance_weights_closed_form(oracle, l):
    """Exact-model transmission weight 2 pi N_l int_0^1 P_l(u) u du (Gauss-Legendre) against the
    closed form: 1/2 (l=0), 1/3 (l=1), and for l >= 2 the standard moment formula."""
    n, L = 3, 5
    N, C = n ** 3, (L + 1) ** 2
    out = np.zeros((N, C), np.complex128)
    r = ((n - 1) * n + 1) * n + 1  # top layer, centre pixel
    out[r, l * l + l] = 1.0
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.8, 1.0, 10.0)
    tr, _ = oracle.images(p, np.zeros(N), np.zeros(N), out, 0, with_ballistic=0)
    from math import factorial
    # int_0^1 P_l(u) u du
    if l == 0:
        m = 0.5
    elif l == 1:
        m = 1.0 / 3.0
    elif l % 2 == 1:
        m = 0.0
    else:
        k = l // 2  # for even l >= 2: (-1)^(k+1) (l-2)! / (2^l (k-1)! (k+1)!)
        m = (-1) ** (k + 1) * factorial(l - 2) / (2 ** l * factorial(k - 1) * factorial(k + 1))
    expect = 2 * np.pi * 0.1 * 0.1 * np.sqrt((2 * l + 1) / (4 * np.pi)) * m
    assert abs(tr[1, 1].real - expect) < 1e-15


@pytest.mark.parametrize("L", [1, 3])
def test_photon_number_without_absorption(rte, oracle, L):
    """ComputePhotonNumber (CPU package/src/Dist.c:538-989, the library's rte_cpu_face_outputs) on the
    oracle's converged CPU-package solve: with mu_a = 0 every photon of the unit beam leaves through
    the faces, up to the discretisation error of the angular truncation and the face quadratures
    (within 10 %); absorption lowers the count monotonically."""
    n = 9
    N, lo, hi = n ** 3, -0.45, 0.45
    p = oracle.params(n, n, n, 0.1, 0.1, 0.1, L, 0.8, 1.0, 10.0, mode=oracle.MODE_CPU, x_min=lo, y_min=lo)
    src = rte.Source(diam=0.1, kind=rte.SRC_CPU)
    counts = []
    for mua in (0.0, 0.01, 0.1, 0.5):
        r = oracle.forward(p, np.full(N, mua), np.full(N, 1.0), src_kind=oracle.SRC_CPU, img_mode=2,
                           stop_rule=oracle.STOP_REL_L2, max_terms=200, tol=1e-12, diam=0.1)
        _, ph = rte.rte.cpu_face_outputs(r["out"], n, n, n, L, lo, hi, lo, hi, 0.0, n * 0.1, src, mua + 1.0)
        assert abs(ph.imag) < 1e-12
        counts.append(ph.real)
    assert abs(counts[0] - 1.0) < 0.1
    assert all(b < a for a, b in zip(counts, counts[1:]))
