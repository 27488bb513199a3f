"""CPU oracle for the fastPLS fit/predict hot path.

TEST INFRASTRUCTURE ONLY.  This package restates, in numpy/scipy (LAPACK from
the OpenBLAS bundled with scipy) plus a g++-compiled libstdc++ RNG helper, the
reference CPU backend of fastPLS (R package tkcaccia/fastPLS, src/fastPLS.cpp,
src/svd_cpu_*.cpp, R/main.R).  Every function cites the reference file:line it
follows.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` may import it, and only as the checker or the timed CPU
baseline.  The product library (``fastpls_b200``) never calls into it and has
no CPU fallback.

Parity pinning: the reference (R + Rcpp + RcppArmadillo) cannot be built or
run in this environment and its test-suite holds no golden vectors, so this
oracle is pinned against (a) the C++ standard's mt19937 known answer, (b) the
reference tests' algebraic identities (prediction identity at 1e-12, PLSSVD
optimized-vs-legacy at 1e-8, LDA projected-vs-explicit at 1e-12, exact
truncated SVD vs a full SVD at 1e-8) and (c) closed-form known-answer cases
(rank-k inputs with exact singular values, one-hot class sums vs dense
products).  Parity against outputs of the reference binary itself is
unpinned.
"""

from .rng import gaussian_matrix, mt19937_raw  # noqa: F401

