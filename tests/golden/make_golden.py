"""Golden fixtures of the CPU oracle (test infrastructure).

    python tests/golden/make_golden.py            # rewrites tests/golden/*.npz

Every fixture holds the inputs of one case (keys ``in_*``, stored exactly) and
the oracle's outputs on them.  The reference (an R package over Armadillo)
cannot be built in this image and its own tests hold no golden vectors, so the
fixtures pin the oracle's restatement against later drift and give the GPU
tests committed expected values:

  c1  SIMPLS regression at its full shape (500 x 2000, rank-20 signal
      s_i = 10 0.8^i + 0.1 noise, 5 responses, rows 1-400 train / 401-500
      test): fast SIMPLS (pls_model2_fast, fastPLS.cpp:2454-2778), classic
      SIMPLS with exact leading vectors (pls_model2 svd_method 3,
      fastPLS.cpp:2260-2451) and PLSSVD (pls_model1, fastPLS.cpp:4780-4986),
      ncomp 5 and 10, seed 1.  X and Y are rounded to multiples of 2^-12 so
      the fixture stores them exactly as int16.
  c2  PLSSVD PLS-DA + LDA, scaled (800 + 200 rows, 200 features, 40 uniform
      classes, class means N(0, 0.5^2), FP32 storage): rSVD (oversample 10,
      power 2, seed 1), LDA on the projected scores (fastPLS.cpp:1930-1957)
      and its predictions (fastPLS.cpp:2100-2147).
  c3  label-aware PLSSVD + candidate kNN, scaled (3000 + 100 rows, 32
      features, 40 Zipf(1.1) classes, normalised prototypes + N(0, 0.3^2)):
      R/main.R:513-655 and fastPLS.cpp:1322-1467 (k 10, tau 0.2, alpha 0.75,
      top_m 20, top 5).
  c4  double CV of SIMPLS PLS-DA, scaled (240 x 600 omics law, 3 x 3 folds,
      ncomp 1..6): fastPLS.cpp:6615-7151 inside pls.double.cv
      (R/main.R:6586-6760), labels and the class scores behind them.
  c5  OPLS filter + Gaussian response compression + SIMPLS, scaled (300 + 60
      rows, 200 features, 150 responses -> 10, north 2, ncomp 3 and 8):
      fastPLS.cpp:4377-4483, R/main.R:1968-2104.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

Q12 = 2.0 ** -12


def _q12(a):
    """Values rounded to multiples of 2^-12 (exact as int16 * 2^-12)."""
    q = np.rint(np.asarray(a, dtype=np.float64) / Q12)
    assert np.all(np.abs(q) < 32767)
    return q.astype(np.int16)


def inputs_of(fx):
    """Fixture dict -> input arrays in their working types."""
    out = {}
    for k, v in fx.items():
        if not k.startswith("in_"):
            continue
        name = k[3:]
        if name.endswith("_q12"):
            out[name[:-4]] = np.asfortranarray(v.astype(np.float64) * Q12)
        else:
            out[name] = np.asfortranarray(v) if v.ndim == 2 else v
    return out


# ---------------------------------------------------------------- inputs

def c1_inputs():
    from fastpls_b200 import synthetic
    d = synthetic.c1_simpls_regression(seed=1)
    X = np.vstack([d["Xtrain"], d["Xtest"]])
    Y = np.vstack([d["Ytrain"], d["Ytest"]])
    return dict(in_X_q12=_q12(X), in_Y_q12=_q12(Y))


def c2_inputs():
    from fastpls_b200 import synthetic
    d = synthetic.c2_plsda(seed=3, n=800, n_test=200, p=200, n_classes=40)
    return dict(in_Xtrain=d["Xtrain"], in_ytrain=d["ytrain"], in_Xtest=d["Xtest"], in_ytest=d["ytest"],
                in_n_classes=np.int32(40))


def c3_inputs():
    rng = np.random.default_rng(7)
    n, nt, p, m = 3000, 100, 32, 40
    pr = 1.0 / np.arange(1, m + 1) ** 1.1
    pr /= pr.sum()
    y = rng.choice(m, size=n + nt, p=pr) + 1
    y[:m] = np.arange(1, m + 1)  # every class has training rows
    proto = rng.standard_normal((m, p)).astype(np.float32)
    proto /= np.linalg.norm(proto, axis=1, keepdims=True)
    X = proto[y - 1] + np.float32(0.3) * rng.standard_normal((n + nt, p), dtype=np.float32)
    X /= np.linalg.norm(X, axis=1, keepdims=True)
    return dict(in_Xtrain=np.asfortranarray(X[:n]), in_ytrain=y[:n].astype(np.int32),
                in_Xtest=np.asfortranarray(X[n:]), in_n_classes=np.int32(m))


def c4_inputs():
    from fastpls_b200 import synthetic
    from fastpls_b200.folds import double_cv_folds
    d = synthetic.c4_omics(seed=2, n=240, p=600, n_informative=20)
    outer, inner = double_cv_folds(d["y"], d["groups"], 3, 3, seed=5)
    return dict(in_X=d["X"], in_y=d["y"], in_outer=outer.astype(np.int32), in_inner=inner.astype(np.int32),
                in_n_classes=np.int32(d["n_classes"]))


def c5_inputs():
    from fastpls_b200 import synthetic
    d = synthetic.c5_lowrank(seed=4, n=300, p=200, q=150, rank=8, n_test=60)
    rng = np.random.default_rng(11)
    G = rng.standard_normal((150, 10)) / np.sqrt(10.0)
    return dict(in_Xtrain=d["Xtrain"], in_Ytrain=d["Ytrain"], in_Xtest=d["Xtest"], in_G=G)


# ---------------------------------------------------------------- oracle runs

C1_NCOMP = [5, 10]
C2_NCOMP = [5, 15]
C5_NCOMP = [3, 8]


def c1_run(x):
    from oracle import pls as opls
    X, Y = x["X"], x["Y"]
    Xtr, Ytr, Xte = X[:400], Y[:400], X[400:]
    out = {}
    fast = opls.pls_model2_fast(Xtr, Ytr, C1_NCOMP, fit=True, seed=1)
    out["fast_B"] = fast["B"]
    out["fast_R"] = fast["R"]
    out["fast_Yfit"] = fast["Yfit"]
    out["fast_R2Y"] = np.asarray(fast["R2Y"], dtype=np.float64)
    out["fast_Ypred"] = opls.pls_predict(fast, Xte, use_B=True)["Ypred"]
    classic = opls.pls_model2(Xtr, Ytr, C1_NCOMP, svd_method=3, seed=1)
    out["classic_B"] = classic["B"]
    out["classic_Ypred"] = opls.pls_predict(classic, Xte, use_B=True)["Ypred"]
    svd = opls.pls_model1(Xtr, Ytr, C1_NCOMP, svd_method=4, seed=1)
    out["plssvd_B"] = svd["B"]
    out["plssvd_Ypred"] = opls.pls_predict(svd, Xte, use_B=True)["Ypred"]
    return out


def c2_run(x):
    from oracle import lda as olda
    from oracle import pls as opls
    m = int(x["n_classes"])
    X = x["Xtrain"].astype(np.float64)
    Xt = x["Xtest"].astype(np.float64)
    model = opls.pls_model1(X, opls.transformy(x["ytrain"]), C2_NCOMP, svd_method=4, rsvd_oversample=10,
                            rsvd_power=2, seed=1)
    out = dict(Ypred=opls.pls_predict(model, Xt, use_B=True)["Ypred"])
    Rp = model["R"] / model["vX"].T
    off = (model["mX"] @ Rp).ravel()
    lda = olda.lda_project_train_prefix(X, Rp, off, x["ytrain"], m, C2_NCOMP, ridge=1e-8)
    for kk in C2_NCOMP:
        lab, sc = olda.lda_project_predict(Xt, Rp[:, :kk], off[:kk], lda[str(kk)], return_scores=True)
        out[f"lda{kk}_linear"] = lda[str(kk)]["linear"]
        out[f"lda{kk}_constants"] = np.asarray(lda[str(kk)]["constants"])
        out[f"lda{kk}_pred"] = np.asarray(lab, dtype=np.int32)
        out[f"lda{kk}_scores"] = sc
    return out


def c3_run(x):
    from oracle import cknn as ok
    from oracle import label_aware as ola
    m = int(x["n_classes"])
    X = x["Xtrain"].astype(np.float64)
    Xt = x["Xtest"].astype(np.float64)
    y = x["ytrain"]
    fit = ola.label_aware_plssvd(X, y, m, [16], svd_method=3)
    C = fit["C_latent"][:, :, 0]
    Tn = ok.row_l2((((X - fit["mX"]) / fit["vX"]) @ fit["R"]) @ C)
    cents = ok.centroids(Tn, y, m)
    Tt = ok.row_l2((((Xt - fit["mX"]) / fit["vX"]) @ fit["R"]) @ C)
    r = ok.candidate_knn_predict(Tt, Tn, y, cents, top_k=5, top_m=20, knn_k=10, tau=0.2, alpha=0.75)
    return dict(W_latent=fit["W_latent"][:, :, 0], top_index=np.asarray(r["top_index"], dtype=np.int32),
                top_score=np.asarray(r["top_score"], dtype=np.float64))


def c4_run(x):
    from oracle import cv as ocv
    r = ocv.double_cv(x["X"].astype(np.float64), x["y"], x["outer"], x["inner"], np.arange(1, 7),
                      int(x["n_classes"]), seed=1)
    return dict(best_comp=r["best_comp"], inner_accuracy=r["inner_accuracy"], pred=r["pred"],
                inner_pred=r["inner_pred"], inner_score=r["inner_score"], outer_score=r["outer_score"])


def c5_run(x):
    from oracle import gaussian_y as og
    from oracle import opls as oopls
    from oracle import pls as opls
    X = x["Xtrain"].astype(np.float64)
    Y = x["Ytrain"].astype(np.float64)
    Xt = x["Xtest"].astype(np.float64)
    filt = oopls.opls_filter(X, Y, 2)
    enc = og.prepare_regression(Y, x["G"])
    model = opls.pls_model2_fast(filt["X"], enc["Z"], C5_NCOMP, seed=1)
    Xtf = oopls.opls_apply_filter(Xt, filt["mX"], filt["vX"], filt["W_orth"], filt["P_orth"])
    Zp = opls.pls_predict(model, Xtf, use_B=True)["Ypred"]
    Yp = np.stack([og.decode_regression(Zp[:, :, a], enc["decoder"], enc["y_center"])
                   for a in range(Zp.shape[2])], axis=2)
    return dict(W_orth=filt["W_orth"], P_orth=filt["P_orth"], decoder=enc["decoder"], Zpred=Zp, Ypred=Yp)


CASES = {
    "c1_simpls_regression": (c1_inputs, c1_run),
    "c2_plssvd_lda": (c2_inputs, c2_run),
    "c3_label_aware_cknn": (c3_inputs, c3_run),
    "c4_double_cv": (c4_inputs, c4_run),
    "c5_opls_gaussian_y": (c5_inputs, c5_run),
}


def main():
    for name, (make, run) in CASES.items():
        fx = make()
        outs = run(inputs_of(fx))
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fx, **outs)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
