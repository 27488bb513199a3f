"""Truncated SVD restatement (test infrastructure only).

Follows the reference CPU SVD layer step for step:
  * truncated_svd dispatch          src/svd_iface.cpp:58-116
  * truncated_svd_cpu_exact         src/svd_cpu_exact.cpp:7-40
  * truncated_svd_cpu_rsvd          src/svd_cpu_rsvd.cpp:95-126
  * finalize_rsvd_from_sample       src/svd_cpu_rsvd.cpp:26-93
LAPACK routines map to the ones Armadillo calls: qr_econ -> geqrf+orgqr,
eig_sym -> syevd, svd_econ(..,"both") -> gesdd, svd_econ(..,"left") -> gesvd.
"""
import numpy as np
import scipy.linalg as sla

from .rng import gaussian_matrix

SVD_METHOD_IRLBA = 1
SVD_METHOD_CPU_EXACT = 3
SVD_METHOD_CPU_RSVD = 4
SVD_METHOD_CUDA_RSVD = 5

EPS = np.finfo(np.float64).eps


def qr_econ_q(Y):
    """Q of the economic Householder QR (geqrf + orgqr), as arma::qr_econ."""
    Q, _ = sla.qr(np.asarray(Y, dtype=np.float64), mode="economic")
    return Q


def svd_econ(A, left_only):
    """arma::svd_econ: gesvd for mode "left", gesdd for mode "both"."""
    driver = "gesvd" if left_only else "gesdd"
    U, s, Vt = sla.svd(np.asarray(A, dtype=np.float64), full_matrices=False,
                       lapack_driver=driver)
    return U, s, Vt.T


def eig_sym_desc(G):
    """arma::eig_sym (syevd) followed by sort_index(.., "descend")."""
    evals, evecs = sla.eigh(G, driver="evd")
    order = np.argsort(-evals, kind="stable")
    return evals[order], evecs[:, order]


class SVDResult:
    def __init__(self, U, s, Vt):
        self.U = U
        self.s = s
        self.Vt = Vt


def truncated_svd_cpu_exact(A, k, left_only=False):
    """src/svd_cpu_exact.cpp:7-40."""
    max_rank = min(A.shape)
    rank = min(max_rank, max(int(k), 1))
    if rank == 0:
        return SVDResult(np.zeros((A.shape[0], 0)), np.zeros(0), np.zeros((0, A.shape[1])))
    U, s, V = svd_econ(A, left_only)
    Vt = None if left_only else V[:, :rank].T.copy()
    return SVDResult(U[:, :rank].copy(), s[:rank].copy(), Vt)


def finalize_rsvd_from_sample(A, Y, k, left_only=False):
    """src/svd_cpu_rsvd.cpp:26-93."""
    max_rank = min(A.shape)
    rank = min(max_rank, max(int(k), 1))
    Q = qr_econ_q(Y)
    B = Q.T @ A
    if B.shape[0] <= B.shape[1]:
        evals_desc, Uhat_desc = eig_sym_desc(B @ B.T)
        tol = EPS * float(max(B.shape)) * (max(evals_desc[0], 1.0) if evals_desc.size else 1.0)
        usable = 0
        while usable < evals_desc.size and evals_desc[usable] > tol:
            usable += 1
        usable = min(usable, rank)
        if usable > 0:
            s = np.sqrt(np.clip(evals_desc[:usable], 0.0, np.inf))
            Uhat = Uhat_desc[:, :usable]
            U = Q @ Uhat
            Vt = None
            if not left_only:
                Vt = (Uhat.T @ B) / s[:, None]
            return SVDResult(U, s, Vt)
    Uhat, s, V = svd_econ(B, left_only)
    U = Q @ Uhat
    Vt = None if left_only else V[:, :rank].T.copy()
    return SVDResult(U[:, :rank].copy(), s[:rank].copy(), Vt)


def rsvd_sample(A, l, power_iters, seed):
    """Range sample of src/svd_cpu_rsvd.cpp:107-121 (sketch + power loop)."""
    Omega = gaussian_matrix(A.shape[1], l, seed)
    Y = A @ Omega
    power_iters = max(int(power_iters), 0)
    if power_iters == 1:
        Y = A @ (A.T @ Y)
    else:
        for _ in range(power_iters):
            Z = A.T @ Y
            Qz = qr_econ_q(Z)
            Y = A @ Qz
    return Y


def truncated_svd_cpu_rsvd(A, k, oversample=10, power_iters=1, seed=1, left_only=False):
    """src/svd_cpu_rsvd.cpp:95-126."""
    max_rank = min(A.shape)
    target = min(max_rank, max(int(k), 1))
    l = min(max_rank, target + max(int(oversample), 0))
    if l >= max_rank:
        return truncated_svd_cpu_exact(A, target, left_only)
    Y = rsvd_sample(A, l, power_iters, seed)
    return finalize_rsvd_from_sample(A, Y, target, left_only)


def truncated_svd(A, k, svd_method=SVD_METHOD_CPU_RSVD, oversample=10, power_iters=1,
                  seed=1, left_only=False, use_full_svd=False):
    """Dispatch of src/svd_iface.cpp:58-116 (method ids: svd_iface.h:39-44).

    The CUDA rSVD id (5) follows the CPU recipe here: the drop-in's parity
    target is the CPU backend.  IRLBA (id 1) needs R's RNG and is not part of
    the GPU path; it raises.
    """
    A = np.asarray(A, dtype=np.float64)
    if k < 1:
        raise ValueError("truncated_svd: k must be >= 1")
    min_dim = min(A.shape)
    force_exact = use_full_svd and svd_method != SVD_METHOD_IRLBA
    if force_exact or min_dim < 6:
        return truncated_svd_cpu_exact(A, k, left_only)
    if svd_method == SVD_METHOD_IRLBA:
        raise NotImplementedError("IRLBA is a CPU-only method outside the GPU path")
    if svd_method in (SVD_METHOD_CPU_RSVD, SVD_METHOD_CUDA_RSVD):
        return truncated_svd_cpu_rsvd(A, k, oversample, power_iters, seed, left_only)
    return truncated_svd_cpu_exact(A, k, left_only)
