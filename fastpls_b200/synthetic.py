"""Seeded synthetic workloads with the shapes and laws of the benchmark configs.

  c1  SIMPLS regression 500 x 2000 (rank-20 signal, s_i = 10*0.8^i), 5 responses
  c2  PLS-DA 20000 x 5000, 100 uniform classes, class means ~ N(0, 0.5^2)
  c3  1.2M x 768 L2-normalised prototypes + N(0, 0.3^2) noise, 1000 Zipf(1.1) classes
  c4  omics 3000 x 20000 log1p(lognormal) centred, 4 classes 40/30/20/10 %,
      50 informative features shifted by 0.5 sd per class
  c5  50000 x 20000 rank-40 signal (s_i = 20*0.9^i) + N(0,1), Y 50000 x 5000

Every generator takes a ``scale`` in (0, 1] that shrinks the row/column counts
for parity tests; scale=1 gives the benchmark shapes.  Data is generated with
numpy's PCG64 from the seed; "stored FP32" configs return float32 arrays.
"""
import numpy as np


def _orth(rng, n, k):
    q, _ = np.linalg.qr(rng.standard_normal((n, k)))
    return q


def c1_simpls_regression(seed=1, n=500, p=2000, m=5, rank=20):
    rng = np.random.default_rng(seed)
    U = _orth(rng, n, rank)
    V = _orth(rng, p, rank)
    s = 10.0 * 0.8 ** np.arange(rank)
    X = (U * s) @ V.T + 0.1 * rng.standard_normal((n, p))
    Bs = rng.standard_normal((p, m)) / np.sqrt(p)
    Y = X @ Bs + 0.05 * rng.standard_normal((n, m))
    ntr = int(round(0.8 * n))
    return dict(Xtrain=np.asfortranarray(X[:ntr]), Ytrain=np.asfortranarray(Y[:ntr]),
                Xtest=np.asfortranarray(X[ntr:]), Ytest=np.asfortranarray(Y[ntr:]))


def c2_plsda(seed=1, n=20000, n_test=5000, p=5000, n_classes=100):
    rng = np.random.default_rng(seed)
    mu = 0.5 * rng.standard_normal((n_classes, p)).astype(np.float32)
    ytot = rng.permutation(np.arange(n + n_test) % n_classes)
    X = mu[ytot] + rng.standard_normal((n + n_test, p), dtype=np.float32)
    y = (ytot + 1).astype(np.int32)
    return dict(Xtrain=np.asfortranarray(X[:n]), ytrain=y[:n], Xtest=np.asfortranarray(X[n:]),
                ytest=y[n:], n_classes=n_classes)


def zipf_labels(rng, n, n_classes, a=1.1):
    w = 1.0 / np.arange(1, n_classes + 1) ** a
    w /= w.sum()
    return rng.choice(n_classes, size=n, p=w)


def c3_prototypes(seed=1, n=1_200_000, n_test=50_000, p=768, n_classes=1000):
    rng = np.random.default_rng(seed)
    proto = rng.standard_normal((n_classes, p)).astype(np.float32)
    proto /= np.linalg.norm(proto, axis=1, keepdims=True)
    y = zipf_labels(rng, n + n_test, n_classes)
    X = proto[y] + 0.3 * rng.standard_normal((n + n_test, p), dtype=np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    y = (y + 1).astype(np.int32)
    return dict(Xtrain=np.asfortranarray(X[:n]), ytrain=y[:n], Xtest=np.asfortranarray(X[n:]),
                ytest=y[n:], n_classes=n_classes)


def c4_omics(seed=1, n=3000, p=20000, n_informative=50, props=(0.4, 0.3, 0.2, 0.1)):
    rng = np.random.default_rng(seed)
    counts = np.floor(np.asarray(props) * n).astype(int)
    counts[0] += n - counts.sum()
    y = rng.permutation(np.repeat(np.arange(len(props)), counts))
    X = np.log1p(np.exp(rng.standard_normal((n, p), dtype=np.float32)))
    sd = X.std(axis=0)
    inf = rng.choice(p, size=n_informative, replace=False)
    X[:, inf] += (0.5 * sd[inf])[None, :] * y[:, None].astype(np.float32)
    X -= X.mean(axis=0, keepdims=True)
    # group ids of 1..5 samples (uneven folds), as the constrain vector
    sizes = []
    while sum(sizes) < n:
        sizes.append(int(rng.integers(1, 6)))
    sizes[-1] -= sum(sizes) - n
    groups = np.repeat(np.arange(1, len(sizes) + 1), sizes)
    return dict(X=np.asfortranarray(X.astype(np.float32)), y=(y + 1).astype(np.int32),
                groups=groups.astype(np.int32), n_classes=len(props))


def c4_double_cv(seed=1, small=False):
    """The double-CV benchmark workload: c4_omics (1500 x 8000 when small) with
    10 outer x 5 inner stratified group folds and the ncomp grid 1..30."""
    from .folds import double_cv_folds
    d = c4_omics(seed=seed, n=1500, p=8000) if small else c4_omics(seed=seed)
    d["outer"], d["inner"] = double_cv_folds(d["y"], d["groups"], 10, 5, seed=seed)
    d["ncomp"] = np.arange(1, 31, dtype=np.int32)
    return d


def c5_lowrank(seed=1, n=50000, p=20000, q=5000, rank=40, n_test=10000):
    rng = np.random.default_rng(seed)
    nt = n + n_test
    U = _orth(rng, nt, rank).astype(np.float32)
    V = _orth(rng, p, rank).astype(np.float32)
    s = (20.0 * 0.9 ** np.arange(rank)).astype(np.float32)
    X = (U * s) @ V.T + rng.standard_normal((nt, p), dtype=np.float32)
    # B* = B1 B2 / sqrt(p rank) has rank 40; Y = (X B1) B2 never forms the p x q product
    B1 = rng.standard_normal((p, rank), dtype=np.float32)
    B2 = rng.standard_normal((rank, q), dtype=np.float32) / np.float32(np.sqrt(p * rank))
    Y = (X @ B1) @ B2 + 0.1 * rng.standard_normal((nt, q), dtype=np.float32)
    return dict(Xtrain=np.asfortranarray(X[:n]), Ytrain=np.asfortranarray(Y[:n]),
                Xtest=np.asfortranarray(X[n:]), Ytest=np.asfortranarray(Y[n:]))
