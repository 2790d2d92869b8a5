"""Seeded synthetic stand-ins for the benchmark matrices (no dataset is read).

Each generator returns a dict with train / test COO arrays in the sampler's input format:
  rows, cols, vals (train), trows, tcols, tvals (test), shape, and for side information
  side = (rows, cols, None, shape) of a binary feature matrix.

  bpmf_uniform  2,000 x 1,500 matrix, 60,000 unique uniform positions, rank-10 U V^T + N(0, 0.5^2),
                10% holdout (the CPU-scale BPMF case; K = 10, alpha = 4).
  bpmf_powerlaw 138,000 x 27,000 matrix, 20M observations; row and column degrees from the
                truncated power law p(k) ~ 1/k on [5, 20000] (inverse CDF), rescaled to the target
                total and clipped to [5, 20000], paired by a configuration model (duplicate
                (i, j) pairs dropped, then topped up to 20M unique cells with extra pairs drawn
                in proportion to the degrees); rank-32 U V^T + N(0, 0.8^2) shifted to mean 3.5, rounded to
                0.5 steps in [0.5, 5]; 10% holdout (K = 32, alpha = 2).  Same shape as the public
                MovieLens-20M rating matrix, generated synthetically.
  macau_side    20,000 x 500 matrix, 1M observations, rank-32 signal + N(0, 1) standardised to mean
                6 / std 1.5; binary side information F (20,000 x 32,768) with Poisson(50) ones per
                row at Zipf(1.1) column indices; true beta ~ N(0, 0.1^2) mixed into U (K = 32).
All sizes take a `scale` so tests can build small versions with the same distributions.
"""
import numpy as np


def _holdout(rng, r, c, v, frac):
    perm = rng.permutation(len(v))
    nt = int(round(len(v) * frac))
    te, tr = perm[:nt], perm[nt:]
    return r[tr], c[tr], v[tr], r[te], c[te], v[te]


def _rowdot(U, V, r, c, chunk=1 << 21):
    out = np.empty(len(r))
    for s in range(0, len(r), chunk):
        e = min(len(r), s + chunk)
        out[s:e] = np.einsum("ij,ij->i", U[r[s:e]], V[c[s:e]])
    return out


def bpmf_uniform(nrow=2000, ncol=1500, nobs=60000, rank=10, noise=0.5, holdout=0.1, seed=0):
    rng = np.random.default_rng(seed)
    pos = rng.choice(nrow * ncol, size=nobs, replace=False)
    r = (pos // ncol).astype(np.int32)
    c = (pos % ncol).astype(np.int32)
    sd = 1.0 / np.sqrt(rank)
    U = rng.normal(0.0, sd, size=(nrow, rank))
    V = rng.normal(0.0, sd, size=(ncol, rank))
    v = _rowdot(U, V, r, c) + rng.normal(0.0, noise, size=nobs)
    tr = _holdout(rng, r, c, v, holdout)
    return dict(rows=tr[0], cols=tr[1], vals=tr[2], trows=tr[3], tcols=tr[4], tvals=tr[5],
                shape=(nrow, ncol), name=f"bpmf_uniform {nrow}x{ncol} nnz={nobs}")


def _powerlaw_degrees(rng, n, total, lo=5, hi=20000):
    # inverse CDF of p(k) ~ 1/k on [lo, hi]: k = lo * (hi/lo)^u
    d = np.floor(lo * (hi / lo) ** rng.random(n)).astype(np.float64)
    scale = total / d.sum()
    for _ in range(50):
        x = np.clip(np.round(d * scale), lo, hi)
        s = x.sum()
        if abs(s - total) <= 0.0005 * total:
            break
        scale *= total / s
    x = x.astype(np.int64)
    diff = int(total - x.sum())
    order = np.argsort(-x, kind="stable")
    i = 0
    while diff != 0:  # spread the remainder over the largest degrees within [lo, hi]
        k = order[i % n]
        step = 1 if diff > 0 else -1
        if lo <= x[k] + step <= hi:
            x[k] += step
            diff -= step
        i += 1
    return x


def bpmf_powerlaw(nrow=138000, ncol=27000, nobs=20_000_000, rank=32, noise=0.8, holdout=0.1,
                  seed=2, scale=1.0):
    rng = np.random.default_rng(seed)
    nrow = max(8, int(nrow * scale))
    ncol = max(8, int(ncol * scale))
    nobs = max(64, int(nobs * scale))
    hi = max(8, int(20000 * min(1.0, scale ** 0.5)))
    dr = _powerlaw_degrees(rng, nrow, nobs, 5, min(hi, ncol))
    dc = _powerlaw_degrees(rng, ncol, nobs, 5, min(hi, nrow))
    rs = np.repeat(np.arange(nrow, dtype=np.int64), dr)
    cs = np.repeat(np.arange(ncol, dtype=np.int64), dc)
    rng.shuffle(cs)
    key = np.unique(rs * ncol + cs)
    # the pairing repeats some (i, j); top up to nobs unique cells with extra pairs drawn in
    # proportion to the row and column degrees
    pr, pc = dr / dr.sum(), dc / dc.sum()
    while len(key) < nobs:
        m = int((nobs - len(key)) * 1.1) + 16
        extra = rng.choice(nrow, size=m, p=pr) * ncol + rng.choice(ncol, size=m, p=pc)
        extra = np.setdiff1d(np.unique(extra), key, assume_unique=True)
        extra = rng.permutation(extra)[:nobs - len(key)]
        key = np.union1d(key, extra)
    r = (key // ncol).astype(np.int32)
    c = (key % ncol).astype(np.int32)
    sd = rank ** -0.25
    U = rng.normal(0.0, sd, size=(nrow, rank))
    V = rng.normal(0.0, sd, size=(ncol, rank))
    v = _rowdot(U, V, r, c) + rng.normal(0.0, noise, size=len(r)) + 3.5
    v = np.clip(np.round(v * 2.0) / 2.0, 0.5, 5.0)
    tr = _holdout(rng, r, c, v, holdout)
    return dict(rows=tr[0], cols=tr[1], vals=tr[2], trows=tr[3], tcols=tr[4], tvals=tr[5],
                shape=(nrow, ncol), name=f"bpmf_powerlaw {nrow}x{ncol} nnz={len(r)}")


def macau_side(nrow=20000, ncol=500, nobs=1_000_000, nfeat=32768, rank=32, ones=50,
               zipf_a=1.1, holdout=0.1, seed=3, scale=1.0):
    rng = np.random.default_rng(seed)
    nrow = max(8, int(nrow * scale))
    nfeat = max(8, int(nfeat * scale))
    nobs = max(64, min(int(nobs * scale), nrow * ncol // 2))
    pos = rng.choice(nrow * ncol, size=nobs, replace=False)
    r = (pos // ncol).astype(np.int32)
    c = (pos % ncol).astype(np.int32)
    # side information: Poisson(ones) entries per row at Zipf(a) column ranks < nfeat
    cnt = rng.poisson(ones, size=nrow)
    tot = int(cnt.sum())
    cols = np.empty(0, np.int64)
    while len(cols) < tot:
        z = rng.zipf(zipf_a, size=2 * tot)
        cols = np.concatenate([cols, z[z <= nfeat] - 1])
    cols = cols[:tot]
    rows = np.repeat(np.arange(nrow, dtype=np.int64), cnt)
    key = np.unique(rows * nfeat + cols)
    fr = (key // nfeat).astype(np.int32)
    fc = (key % nfeat).astype(np.int32)
    sd = rank ** -0.25
    U = rng.normal(0.0, sd, size=(nrow, rank))
    V = rng.normal(0.0, sd, size=(ncol, rank))
    beta = rng.normal(0.0, 0.1, size=(nfeat, rank))
    Fb = np.zeros((nrow, rank))
    np.add.at(Fb, fr, beta[fc])
    U = U + Fb
    v = _rowdot(U, V, r, c) + rng.normal(0.0, 1.0, size=nobs)
    v = 6.0 + 1.5 * (v - v.mean()) / v.std()
    tr = _holdout(rng, r, c, v, holdout)
    return dict(rows=tr[0], cols=tr[1], vals=tr[2], trows=tr[3], tcols=tr[4], tvals=tr[5],
                shape=(nrow, ncol), side=(fr, fc, None, (nrow, nfeat)),
                name=f"macau_side {nrow}x{ncol} nnz={nobs} F={nrow}x{nfeat} nnzF={len(fr)}")


def batched_uneven(nprob=512, seed0=5000, holdout=0.1, rows=(200, 4000), cols=(100, 1000),
                   density=(0.01, 0.05), ks=(8, 16, 32), noise=0.5):
    """Many independent BPMF problems of uneven size: problem i (numpy seed seed0 + i) has
    U[rows] x U[cols] entries at density U[density] (unique random positions), latent dimension
    drawn from ks, values rank-K U V^T + N(0, noise^2) with U, V ~ N(0, 1/sqrt(K)), and a random
    holdout.  Returns (problems, num_latent, seeds)."""
    problems, Ks, seeds = [], [], []
    for i in range(nprob):
        rng = np.random.default_rng(seed0 + i)
        nr = int(rng.integers(rows[0], rows[1] + 1))
        nc = int(rng.integers(cols[0], cols[1] + 1))
        dens = float(rng.uniform(density[0], density[1]))
        K = int(rng.choice(ks))
        want = max(16, int(nr * nc * dens))
        pos = np.unique(rng.integers(0, nr * nc, size=int(want * 1.1) + 16))
        pos = rng.permutation(pos)[:want]
        r = (pos // nc).astype(np.int32)
        c = (pos % nc).astype(np.int32)
        sd = 1.0 / np.sqrt(K)
        U = rng.normal(0.0, sd, size=(nr, K))
        V = rng.normal(0.0, sd, size=(nc, K))
        v = np.sum(U[r] * V[c], axis=1) + rng.normal(0.0, noise, size=len(r))
        tr = _holdout(rng, r, c, v, holdout)
        problems.append(dict(rows=tr[0], cols=tr[1], vals=tr[2], trows=tr[3], tcols=tr[4],
                             tvals=tr[5], shape=(nr, nc)))
        Ks.append(K)
        seeds.append(seed0 + i)
    return problems, Ks, seeds
