"""The oracle's small dense linear algebra against LAPACK (numpy), FP64.

The reference delegates two decompositions to Eigen, and no reference test pins
them: the 3 x 3 self-adjoint eigensolver behind Stiffness::enforce_spd
(stiffness.cpp:236-254) and the 3 x 2 JacobiSVD of the strain limits
(strain_limiting.cpp:34-37), which the CORRECTED membrane uses too. The
oracle restates both from their definitions (the device kernels run the same
formulas). Here they are checked against an independent implementation of
the same definitions on seeded random, near-degenerate and rank-deficient
inputs: the clamped spectral reconstruction V max(L, eps) V^T, the singular
values and the polar factor U V^T, which are the only quantities the step
uses (eigenvector and singular-vector signs cancel in both).
"""
from __future__ import annotations

import numpy as np
import pytest


def random_symmetric(rng, kind):
    Q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if kind == "generic":
        w = rng.normal(size=3) * 10.0 ** rng.uniform(-3, 3)
    elif kind == "repeated":
        a = rng.normal()
        w = np.array([a, a, rng.normal()])
    elif kind == "spread":
        w = np.array([1e8, 1.0, -1e-3]) * rng.uniform(0.5, 2.0, 3)
    else:                                                  # one eigenvalue at the clamp
        w = np.array([rng.uniform(1, 2), 1e-8, -rng.uniform(1, 2)])
    return (Q * w) @ Q.T


@pytest.mark.parametrize("kind", ["generic", "repeated", "spread", "clamp"])
def test_enforce_spd_is_the_clamped_spectral_reconstruction(oracle, kind):
    O = oracle.f64
    rng = np.random.default_rng(hash(kind) % 2**32)
    for _ in range(100):
        A = random_symmetric(rng, kind)
        S = O.enforce_spd(A)
        w, Q = np.linalg.eigh(A)
        ref = (Q * np.maximum(w, 1e-8)) @ Q.T
        scale = max(np.abs(A).max(), 1e-8)
        np.testing.assert_allclose(S, ref, rtol=0, atol=1e-12 * scale)
        assert np.linalg.eigvalsh(0.5 * (S + S.T)).min() >= 1e-8 * (1 - 1e-6) - 1e-12 * scale


def random_F(rng, kind):
    F = rng.normal(size=(3, 2))
    if kind == "equal":                                    # equal singular values: a scaled isometry
        Q, _ = np.linalg.qr(rng.normal(size=(3, 2)))
        R2, _ = np.linalg.qr(rng.normal(size=(2, 2)))
        F = rng.uniform(0.5, 2.0) * Q @ R2
    elif kind == "near_rank_one":
        u, v = rng.normal(size=3), rng.normal(size=2)
        F = np.outer(u, v) + 1e-7 * rng.normal(size=(3, 2))
    elif kind == "near_identity":                          # the cloth at rest, slightly strained
        Q, _ = np.linalg.qr(rng.normal(size=(3, 2)))
        F = Q @ (np.eye(2) + 1e-3 * rng.normal(size=(2, 2)))
    return F


@pytest.mark.parametrize("kind", ["generic", "equal", "near_rank_one", "near_identity"])
def test_svd32_values_and_polar_factor(oracle, kind):
    O = oracle.f64
    rng = np.random.default_rng(7 + len(kind))
    for _ in range(100):
        F = random_F(rng, kind)
        U, s, V, ok = O.svd32(F)
        assert ok
        Un, sn, Vtn = np.linalg.svd(F, full_matrices=False)
        scale = sn[0]
        np.testing.assert_allclose(V.T @ V, np.eye(2), atol=1e-12)
        assert abs(s[0] - sn[0]) <= 1e-12 * scale
        if kind == "near_rank_one":
            # the singular values come from the eigenvalues of F^T F, so the small one
            # carries an absolute error of about sqrt(eps) s0 (and U's second column
            # is not unit length) once s1 falls below about 1e-4 s0: a face collapsed
            # to a sliver, which the strain limits keep every workload far from
            assert abs(s[1] - max(sn[1], 1e-6)) <= 1e-7 * scale
            continue
        # singular values (both clamped at 1e-6, the reference's kDegenerateThreshold)
        np.testing.assert_allclose(s, np.maximum(sn, 1e-6), rtol=1e-9, atol=1e-12 * scale)
        np.testing.assert_allclose(U.T @ U, np.eye(2), atol=1e-10)
        np.testing.assert_allclose(U @ np.diag(s) @ V.T, F, rtol=0, atol=1e-11 * scale)
        # the polar factor R = U V^T, unique for a full-rank F
        np.testing.assert_allclose(U @ V.T, Un @ Vtn, rtol=0, atol=1e-9 * scale / sn[1])


def test_triplet_assembly_sums_duplicates_like_scipy(oracle):
    """Sparse assembly from triplets (the reference's SparseMatrix::setFromTriplets
    in matrix_assembly.cpp): duplicates summed, columns sorted per row, against
    scipy's COO -> CSR conversion of the same triplets."""
    import scipy.sparse as sp

    O = oracle.f64
    rng = np.random.default_rng(3)
    n = 60
    k = 4000                                               # about one duplicate per entry
    rows = rng.integers(0, n, k)
    cols = rng.integers(0, n, k)
    vals = rng.normal(size=k) * 10.0 ** rng.uniform(-6, 6, k)
    A = O.csr_from_triplets(n, rows, cols, vals)
    B = sp.coo_matrix((vals, (rows, cols)), shape=(n, n)).tocsr()
    B.sum_duplicates()
    B.sort_indices()
    np.testing.assert_array_equal(np.asarray(A["rowptr"]), B.indptr)
    np.testing.assert_array_equal(np.asarray(A["cols"]), B.indices)
    scale = np.abs(vals).max()
    np.testing.assert_allclose(np.asarray(A["vals"]), B.data, rtol=1e-12, atol=1e-15 * scale)
