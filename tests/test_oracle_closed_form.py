"""Checks the oracle's parts that no reference test pins (sample_latent_blas, CondNormalWishart,
MvNormal draws, block-CG at K RHS) against closed forms computed with numpy/scipy on small
cases."""
import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from oracle import oracle as orc


def rand_csr(rng, nrow, ncol, density, vals=True):
    m = sp.random(nrow, ncol, density=density, random_state=rng, format="csr")
    if vals:
        m.data = rng.normal(3.0, 1.0, m.nnz)
    return m


def test_normal_and_gamma_draws_moments():
    z = np.array([orc.normal(7, 3, "row_noise", 1, i, j) for i in range(4000) for j in range(8)])
    assert abs(z.mean()) < 0.02 and abs(z.var() - 1) < 0.03
    g = np.array([orc.gamma(7, s, "wishart_diag", 0, 0, 2.5) for s in range(20000)])
    assert abs(g.mean() - 2.5) < 0.05 and abs(g.var() - 2.5) < 0.15
    g = np.array([orc.gamma(7, s, "wishart_diag", 0, 0, 0.4) for s in range(20000)])
    assert abs(g.mean() - 0.4) < 0.02


def test_sample_latents_matches_numpy_closed_form():
    rng = np.random.default_rng(0)
    K, nrow, ncol = 6, 40, 30
    Y = rand_csr(rng, nrow, ncol, 0.2)
    R = orc.Csr.from_scipy(Y)
    V = rng.normal(size=(ncol, K))
    A = rng.normal(size=(K, K))
    Lam = A @ A.T + K * np.eye(K)
    mu = rng.normal(size=K)
    Uhat = rng.normal(size=(nrow, K))
    z = rng.normal(size=(nrow, K))
    alpha, mean = 2.0, 3.1
    U, st = orc.sample_latents(K, R, V, mean, alpha, mu, Lam, Uhat=Uhat, z=z)
    assert st == 0
    for n in range(nrow):
        cols = Y.indices[Y.indptr[n]:Y.indptr[n + 1]]
        ys = Y.data[Y.indptr[n]:Y.indptr[n + 1]]
        Vn = V[cols]
        MM = Lam + alpha * Vn.T @ Vn
        rr = alpha * Vn.T @ (ys - mean) + Lam @ (mu + Uhat[n])
        L = np.linalg.cholesky(MM)
        x = sla.solve_triangular(L.T, sla.solve_triangular(L, rr, lower=True) + z[n],
                                 lower=False)
        np.testing.assert_allclose(U[n], x, rtol=1e-11, atol=1e-12)


def test_sample_latents_reports_cholesky_failure():
    K = 3
    R = orc.Csr(np.array([0, 0]), np.zeros(0, np.int32), np.zeros(0), 1, 1)
    U, st = orc.sample_latents(K, R, np.zeros((1, K)), 0.0, 1.0, np.zeros(K), -np.eye(K))
    assert st == -1


def test_cond_normal_wishart_moments():
    # Lambda ~ W(T_c, nu_c) has mean nu_c * T_c; mu | Lambda ~ N(mu_c, (kappa_c Lambda)^-1).
    rng = np.random.default_rng(1)
    K, N = 3, 25
    U = rng.normal(size=(N, K)) + np.array([0.5, -1.0, 2.0])
    mu0 = np.zeros(K)
    kappa, nu, T = 2.0, K, np.eye(K)
    NU = U.sum(0)
    mu_c = (kappa * mu0 + NU) / (kappa + N)
    X = T + U.T @ U + kappa * np.outer(mu0, mu0) - (kappa + N) * np.outer(mu_c, mu_c)
    Tc = np.linalg.inv(X)
    lams, mus = [], []
    for s in range(3000):
        mu, Lam, st = orc.cond_normal_wishart(U, mu0, kappa, T, nu, seed=11, sweep=s)
        assert st == 0
        lams.append(Lam)
        mus.append(mu)
    lams = np.array(lams)
    mus = np.array(mus)
    want = (nu + N) * Tc
    np.testing.assert_allclose(lams.mean(0), want, atol=0.06 * np.abs(want).max())
    np.testing.assert_allclose(mus.mean(0), mu_c, atol=0.05)
    assert np.allclose(lams, np.transpose(lams, (0, 2, 1)), atol=1e-12)


def test_blockcg_solves_regularised_normal_equations():
    rng = np.random.default_rng(2)
    nrow, nfeat, nrhs = 200, 120, 7
    F = sp.random(nrow, nfeat, density=0.05, random_state=rng, format="csr")
    F.data[:] = 1.0
    B = rng.normal(size=(nfeat, nrhs))
    reg = 1.5
    Fc, Ftc = orc.Csr.from_scipy(F, True), orc.Csr.from_scipy(F.T, True)
    X, it = orc.blockcg(Fc, Ftc, reg, B, 1e-8)
    A = (F.T @ F).toarray() + reg * np.eye(nfeat)
    np.testing.assert_allclose(X, np.linalg.solve(A, B), rtol=1e-5, atol=1e-6)
    assert 0 < it < 200
    # blocked wrapper with 32+8 blocking on 45 RHS (two blocks)
    B2 = rng.normal(size=(nfeat, 45))
    X2, _ = orc.blockcg(Fc, Ftc, reg, B2, 1e-8, blocksize=32, excess=8)
    np.testing.assert_allclose(X2, np.linalg.solve(A, B2), rtol=1e-5, atol=1e-6)


def test_model_runs_and_learns_small_bpmf():
    rng = np.random.default_rng(3)
    nrow, ncol, K = 120, 80, 4
    Ut = rng.normal(size=(nrow, 3))
    Vt = rng.normal(size=(ncol, 3))
    Yfull = Ut @ Vt.T + rng.normal(scale=0.3, size=(nrow, ncol))
    mask = rng.random((nrow, ncol)) < 0.3
    r, c = np.nonzero(mask)
    test = rng.random(len(r)) < 0.1
    Ytr = sp.coo_matrix((Yfull[r[~test], c[~test]], (r[~test], c[~test])), shape=(nrow, ncol))
    Yte = sp.csc_matrix((Yfull[r[test], c[test]], (r[test], c[test])), shape=(nrow, ncol))
    Yte.sort_indices()
    te = Yte.tocoo()
    m = orc.Model(K, 1.0 / 0.09, 5)
    Rr, Rc = orc.Csr.from_scipy(Ytr), orc.Csr.from_scipy(Ytr.T)
    m.set_train(Rr, Rc, Ytr.tocsc().sum() / Ytr.nnz)
    m.set_test(te.row, te.col, te.data)
    for it in range(60):
        assert m.sweep(it, 30) == 0
    rmse, rmse1 = m.rmse()
    assert rmse < 0.6, rmse


def test_adaptive_noise_matches_closed_form():
    """AdaptiveGaussianNoise (noisemodels.cpp:14-33, 55-81): var_total, the initial and capped
    precision, and the update's Gamma(aN, 1/bN) draw from the squared training residuals."""
    rng = np.random.default_rng(11)
    nrow, ncol, K, seed = 50, 40, 5, 99
    Y = rand_csr(rng, nrow, ncol, 0.25).tocsc()
    Y.sort_indices()
    mean = Y.sum() / Y.nnz
    m = orc.Model(K, 1.0, seed)
    m.set_train(orc.Csr.from_scipy(Y), orc.Csr.from_scipy(Y.T), mean)
    m.set_noise_adaptive(1.0, 10.0)
    var_total = np.mean((Y.data - mean) ** 2)
    alpha, alpha_max, vt = m.noise()
    assert abs(vt - var_total) <= 1e-14 * var_total
    assert abs(alpha - 2.0 / var_total) <= 1e-14 * alpha
    assert abs(alpha_max - 11.0 / var_total) <= 1e-14 * alpha_max
    U = rng.normal(scale=0.5, size=(nrow, K))
    V = rng.normal(scale=0.5, size=(ncol, K))
    m.set("latents", 0, U)
    m.set("latents", 1, V)
    m.update_noise(7)
    Yc = Y.tocoo()
    sse = np.sum((np.sum(U[Yc.row] * V[Yc.col], axis=1) + mean - Yc.data) ** 2)
    aN = 0.5 + Y.nnz / 2.0
    bN = 0.5 * var_total + sse / 2.0
    want = min(orc.gamma(seed, 7, "noise_alpha", 0, 0, aN) / bN, alpha_max)
    assert abs(m.noise()[0] - want) <= 1e-12 * want
    # latents that fit Y exactly: the draw (about nnz / var_total) is capped at alpha_max
    Yc = Y.tocoo()
    a, b = rng.normal(size=nrow), rng.normal(size=ncol)
    ab = a[Yc.row] * b[Yc.col]
    Yx = sp.coo_matrix((ab + 3.0, (Yc.row, Yc.col)), shape=Y.shape).tocsc()
    Yx.sort_indices()
    mx = Yx.sum() / Yx.nnz
    Ux = np.zeros((nrow, K))
    Vx = np.zeros((ncol, K))
    Ux[:, 0], Vx[:, 0] = a, b
    Ux[:, 1], Vx[:, 1] = 1.0, -(mx - 3.0)
    m2 = orc.Model(K, 1.0, seed)
    m2.set_train(orc.Csr.from_scipy(Yx), orc.Csr.from_scipy(Yx.T), mx)
    m2.set_noise_adaptive(1.0, 10.0)
    m2.set("latents", 0, Ux)
    m2.set("latents", 1, Vx)
    m2.update_noise(0)
    assert m2.noise()[0] == m2.noise()[1]


def test_adaptive_noise_model_learns_noise_level():
    """A full adaptive-noise run: the precision settles near 1 / noise variance (signal-to-noise
    below sn_max), like AdaptiveGaussianNoise in MacauX::run (macau.cpp:110-147)."""
    rng = np.random.default_rng(5)
    nrow, ncol, K, sd = 150, 100, 4, 0.8
    Ut = rng.normal(size=(nrow, 3))
    Vt = rng.normal(size=(ncol, 3))
    mask = rng.random((nrow, ncol)) < 0.4
    r, c = np.nonzero(mask)
    v = np.sum(Ut[r] * Vt[c], axis=1) + rng.normal(scale=sd, size=len(r))
    Y = sp.coo_matrix((v, (r, c)), shape=(nrow, ncol)).tocsc()
    Y.sort_indices()
    m = orc.Model(K, 1.0, 3)
    m.set_train(orc.Csr.from_scipy(Y), orc.Csr.from_scipy(Y.T), Y.sum() / Y.nnz)
    m.set_noise_adaptive(1.0, 10.0)
    alphas = []
    for it in range(40):
        assert m.sweep(it, 20) == 0
        alphas.append(m.noise()[0])
    a = np.mean(alphas[20:])
    assert 0.7 / sd**2 < a < 1.5 / sd**2 and a < m.noise()[1], a


def _one_model(rng, nrow, ncol, K, nfeat, seed, lambda_beta=5.0, binary=False):
    Y = rand_csr(rng, nrow, ncol, 0.3).tocsc()
    Y.sort_indices()
    F = sp.random(nrow, nfeat, density=0.5, random_state=rng, format="csr")
    if binary:
        F.data[:] = 1.0
    m = orc.Model(K, 1.5, seed)
    m.set_train(orc.Csr.from_scipy(Y), orc.Csr.from_scipy(Y.T), Y.sum() / Y.nnz)
    m.set_side_one(0, orc.Csr.from_scipy(F, binary), orc.Csr.from_scipy(F.T, binary), lambda_beta)
    return m, Y, F


def test_univariate_row_sampler_targets_the_gaussian_posterior():
    """MacauOnePrior::sample_latents (macauoneprior.cpp:41-95) is a coordinate-wise Gibbs sweep
    on a row's Gaussian posterior: with the other factor and the hyperparameters held fixed,
    its chain's mean and covariance approach P^-1 b and P^-1, P = diag(lambda) + alpha V'V."""
    rng = np.random.default_rng(21)
    K, nrow, ncol = 3, 4, 12
    m, Y, _ = _one_model(rng, nrow, ncol, K, 2, seed=8)
    V = rng.normal(size=(ncol, K))
    m.set("latents", 1, V)
    mu = np.array([0.2, -0.1, 0.3])
    m.set("mu", 0, mu)
    lam = np.array([2.0, 3.0, 1.5])
    m.set("Lambda", 0, np.diag(lam))
    mean = Y.sum() / Y.nnz
    Yr = Y.tocsr()
    draws = []
    for it in range(20000):
        m.sample_mode(0, it)
        draws.append(m.latents(0)[1].copy())
    draws = np.array(draws[200:])
    cols = Yr.indices[Yr.indptr[1]:Yr.indptr[2]]
    vals = Yr.data[Yr.indptr[1]:Yr.indptr[2]]
    Vr = V[cols]
    P = np.diag(lam) + 1.5 * Vr.T @ Vr
    b = lam * mu + 1.5 * Vr.T @ (vals - mean)
    want_mean = np.linalg.solve(P, b)
    want_cov = np.linalg.inv(P)
    sd = np.sqrt(np.diag(want_cov))
    assert np.all(np.abs(draws.mean(0) - want_mean) < 0.05 * sd + 0.01), (draws.mean(0), want_mean)
    np.testing.assert_allclose(np.cov(draws.T), want_cov, atol=0.08 * sd.max() ** 2)


def test_univariate_update_prior_matches_restatement():
    """MacauOnePrior::update_prior (macauoneprior.cpp:189-290) against a numpy restatement on a
    small case: Normal-Wishart of U - Uhat, the feature-by-feature link sampler, Uhat = F beta,
    and the per-dimension lambda_beta draws."""
    rng = np.random.default_rng(4)
    K, nrow, ncol, nfeat, seed, it = 6, 30, 20, 5, 77, 3
    for binary in (False, True):
        m, Y, F = _one_model(rng, nrow, ncol, K, nfeat, seed, lambda_beta=2.5, binary=binary)
        U = rng.normal(size=(nrow, K))
        m.set("latents", 0, U)
        beta0 = rng.normal(scale=0.3, size=(nfeat, K))
        m.set("beta", 0, beta0)
        Uhat0 = F @ beta0
        m.set("uhat", 0, Uhat0)
        lb = np.full(K, 2.5)
        assert m.update_prior(0, it) == 0
        mu, Lam, st = orc.cond_normal_wishart(U - Uhat0, np.zeros(K), 2.0, np.eye(K), K, seed=seed,
                                              sweep=it, mode=0)
        assert st == 0
        np.testing.assert_allclose(m.mu(0), mu, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(m.Lambda(0), Lam, rtol=1e-12, atol=1e-14)
        lam = np.diag(Lam)
        Fc = F.tocsc()
        colsq = np.asarray(Fc.multiply(Fc).sum(axis=0)).ravel()
        beta = beta0.copy()
        Z = U - mu - Uhat0
        for d0 in range(0, K, 4):
            ds = range(d0, min(K, d0 + 4))
            for f in range(nfeat):
                rows = Fc.indices[Fc.indptr[f]:Fc.indptr[f + 1]]
                v = Fc.data[Fc.indptr[f]:Fc.indptr[f + 1]]
                for d in ds:
                    zx = np.dot(v, Z[rows, d])
                    A = lb[d] + lam[d] * colsq[f]
                    B = lam[d] * (zx + beta[f, d] * colsq[f])
                    z = orc.normal(seed, it, "beta_one", 0, f, d)
                    new = B / A + np.sqrt(1.0 / A) * z
                    Z[rows, d] += v * (beta[f, d] - new)
                    beta[f, d] = new
        np.testing.assert_allclose(m.beta(0), beta, rtol=1e-10, atol=1e-12)
        np.testing.assert_allclose(m.uhat(0), F @ beta, rtol=1e-10, atol=1e-12)
        a = 0.1 + nfeat / 2.0
        want = [orc.gamma(seed, it, "lambda_beta", 0, d, a) / (0.1 + np.sum(beta[:, d] ** 2) / 2)
                for d in range(K)]
        np.testing.assert_allclose(m.lambda_beta_one(0), want, rtol=1e-10)


def test_univariate_model_learns_small_matrix():
    """A univariate chain (MacauOnePrior on the rows, BPMF on the columns) learns a low-rank
    matrix about as well as the BPMF chain, like test_macau_univariate (test_macau.py:64-73)."""
    rng = np.random.default_rng(3)
    nrow, ncol, K = 120, 80, 4
    Ut = rng.normal(size=(nrow, 3))
    Vt = rng.normal(size=(ncol, 3))
    Yfull = Ut @ Vt.T + rng.normal(scale=0.3, size=(nrow, ncol))
    mask = rng.random((nrow, ncol)) < 0.3
    r, c = np.nonzero(mask)
    test = rng.random(len(r)) < 0.1
    Ytr = sp.coo_matrix((Yfull[r[~test], c[~test]], (r[~test], c[~test])), shape=(nrow, ncol))
    Yte = sp.csc_matrix((Yfull[r[test], c[test]], (r[test], c[test])), shape=(nrow, ncol))
    Yte.sort_indices()
    te = Yte.tocoo()
    F = sp.csr_matrix(np.hstack([Ut + rng.normal(scale=0.5, size=Ut.shape), np.ones((nrow, 1))]))
    m = orc.Model(K, 1.0 / 0.09, 5)
    m.set_train(orc.Csr.from_scipy(Ytr), orc.Csr.from_scipy(Ytr.T), Ytr.tocsc().sum() / Ytr.nnz)
    m.set_test(te.row, te.col, te.data)
    m.set_side_one(0, orc.Csr.from_scipy(F), orc.Csr.from_scipy(F.T), 5.0)
    for it in range(80):
        assert m.sweep(it, 40) == 0
    rmse, _ = m.rmse()
    assert rmse < 0.6, rmse
    assert np.linalg.norm(m.beta(0)) > 0.1
