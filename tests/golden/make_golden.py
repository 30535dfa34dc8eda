"""Generate tests/golden/*.npz: small cohorts and the outputs of an independent pure-Python /
numpy restatement of the reference's hot path.

The reference (Julia) cannot run here, so these fixtures are not reference outputs; they are
a second restatement written separately from oracle/admix_oracle.c, and the tests require the
C oracle and the GPU engine to agree with them.  Each function cites the reference lines it
follows.  Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import math
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent

G_MAP = np.array([0.0, 0.0, 1.0, 2.0])     # loops.jl:3
NM_MAP = np.array([1.0, 0.0, 1.0, 1.0])    # loops.jl:2


def make_cohort(I, J, K, seed, miss=0.02):
    rng = np.random.default_rng(seed)
    q = rng.gamma(0.5, size=(I, K)); q /= q.sum(1, keepdims=True)
    p = rng.uniform(0.05, 0.95, size=(J, K))
    f = q @ p.T                                    # I x J
    g = rng.binomial(2, f)
    codes = np.where(g == 0, 0, np.where(g == 1, 2, 3)).astype(np.uint8)
    codes[rng.random((I, J)) < miss] = 1
    Ib = (I + 3) // 4
    bed = np.zeros((J, Ib), np.uint8)
    for i in range(I):
        bed[:, i >> 2] |= (codes[i, :] << (2 * (i & 3))).astype(np.uint8)
    return bed, codes


def decode(bed, I):
    J, Ib = bed.shape
    codes = np.empty((I, J), np.uint8)
    for i in range(I):
        codes[i] = (bed[:, i >> 2] >> (2 * (i & 3))) & 3     # loops.jl:529-532
    return G_MAP[codes], NM_MAP[codes]


def loglik(g, nm, q, p):                                      # loops.jl:517-539
    qp = q @ p.T
    return float(np.sum(nm * (g * np.log(qp) + (2 - g) * np.log(1 - qp))))


def grad_hess_q(g, nm, q, p):                                 # loops.jl:867-894
    qp = q @ p.T
    a = nm * g / qp**2; b = nm * (2 - g) / (1 - qp)**2
    H = np.einsum("ij,jk,jl->ikl", a, p, p) + np.einsum("ij,jk,jl->ikl", b, 1 - p, 1 - p)
    z = (nm * g / qp) @ p + (nm * (2 - g) / (1 - qp)) @ (1 - p)
    return H, z


def grad_hess_p(g, nm, q, p):                                 # loops.jl:923-950
    qp = q @ p.T
    w = nm * (g / qp**2 + (2 - g) / (1 - qp)**2)
    H = np.einsum("ij,ik,il->jkl", w, q, q)
    z = (nm * (g / qp - (2 - g) / (1 - qp))).T @ q
    return H, z


def em_q(g, nm, q, p):                                        # loops.jl:610-632, algorithms_inner.jl:89
    qp = q @ p.T
    J = p.shape[0]
    s = (nm * g / qp) @ p + (nm * (2 - g) / (1 - qp)) @ (1 - p)
    return q * s / (2 * J)


def em_p(g, nm, q, p):                                        # loops.jl:700-721, algorithms_inner.jl:133-137
    qp = q @ p.T
    A = p * ((nm * g / qp).T @ q)
    B = (1 - p) * ((nm * (2 - g) / (1 - qp)).T @ q)
    return A / (A + B)


def sweep(A, k, inverse):                                     # qp.jl:297-317
    n = A.shape[0]
    piv = 1.0 / A[k, k]
    tmp = A[:, k].copy()
    A[:, k] = 0.0; A[k, :] = 0.0
    tmp[k] = 1.0 if inverse else -1.0
    for i in range(n):
        pv = piv * tmp[i]
        for j in range(n):
            A[j, i] = A[j, i] - pv * tmp[j]


def create_tableau(H, r, x, simplex):                         # qp.jl:8-76 with mu = 0
    K = H.shape[0]
    n = K + 2 if simplex else K + 1
    T = np.zeros((n, n))
    T[:K, :K] = H
    T[n - 1, :K] = -r; T[:K, n - 1] = -r
    if simplex:
        T[K, :K] = 1.0; T[:K, K] = 1.0
        T[K + 1, K] = T[K, K + 1] = 1.0 - sum(x)
    return T


def quadratic_program(T, par, p, c):                          # qp.jl:171-292, pmin 0, pmax 1
    n = p + c + 1
    delta = np.zeros(p)
    small, tol = 1e-5, 1e-8
    d = np.diag(T).copy()
    for i in range(p):
        if d[i] <= 0 or T[i, i] < d[i] * tol:
            return 0, delta
        sweep(T, i, False)
    swept = [True] * p
    for i in range(p, p + c):
        if T[i, i] >= 0:
            return 0, delta
        sweep(T, i, False)
    e = n - 1
    for iteration in range(1, 1001):
        a = 1.0
        for i in range(p):
            if swept[i]:
                ui = T[i, e]
                ai = (1.0 - par[i] - delta[i]) if ui > 0 else (0.0 - par[i] - delta[i])
                if abs(ui) > 1e-10:
                    a = min(a, ai / ui)
        for i in range(p):
            if swept[i]:
                ui = T[i, e]
                delta[i] = delta[i] + a * ui
                T[i, e] = (1.0 - a) * ui
                T[e, i] = T[i, e]
        moved = False
        for i in range(p):
            xi = par[i] + delta[i]
            critical = (0.0 >= xi - small) or (1.0 <= xi + small)
            if swept[i] and abs(T[i, i]) > 1e-10 and critical:
                sweep(T, i, True); swept[i] = False; moved = True
                break
        if moved:
            continue
        for i in range(p):
            ui = T[i, e]
            xi = par[i] + delta[i]
            violation = (ui > 0 and 0.0 >= xi - small) or (ui < 0 and 1.0 <= xi + small)
            if not swept[i] and violation:
                sweep(T, i, False); swept[i] = True; moved = True
                break
        if moved:
            continue
        return iteration, delta
    return 0, delta


def project_q(b, pc=1e-5):                                    # projections.jl:27-59
    n = len(b)
    tau = 1.0 - n * pc
    b = b - pc
    s = sorted(b, reverse=True)
    tsum, bget, tmax = 0.0, False, 0.0
    for i in range(n - 1):
        tsum += s[i]
        tmax = (tsum - tau) / (i + 1)
        if tmax >= s[i + 1]:
            bget = True
            break
    if not bget:
        tmax = (tsum + s[n - 1] - tau) / n
    return np.maximum(b - tmax, 0.0) + pc


def project_p(b, pc=1e-5):                                    # projections.jl:69-74
    return np.minimum(np.maximum(b, pc), 1 - pc)


def update_q(g, nm, q, p):                                    # algorithms_inner.jl:167-231
    H, z = grad_hess_q(g, nm, q, p)
    out = np.empty_like(q); st = np.empty(q.shape[0], np.int32)
    for i in range(q.shape[0]):
        T = create_tableau(H[i], -z[i], q[i], True)
        st[i], dlt = quadratic_program(T, q[i], q.shape[1], 1)
        out[i] = project_q(q[i] + dlt)
    return out, st


def update_p(g, nm, q, p):                                    # algorithms_inner.jl:245-310
    H, z = grad_hess_p(g, nm, q, p)
    out = np.empty_like(p); st = np.empty(p.shape[0], np.int32)
    for j in range(p.shape[0]):
        T = create_tableau(H[j], -z[j], p[j], False)
        st[j], dlt = quadratic_program(T, p[j], p.shape[1], 0)
        out[j] = project_p(p[j] + dlt)
    return out, st


def qn_iteration(g, nm, x, ll_prev, U, V, it, Q):           # algorithms_outer.jl:92-159, quasi_newton.jl
    I = g.shape[0]
    q, p = x[:I], x[I:]
    q1, _ = update_q(g, nm, q, p)
    p1, _ = update_p(g, nm, q1, p)
    q2, _ = update_q(g, nm, q1, p1)
    p2, _ = update_p(g, nm, q2, p1)
    x1 = np.vstack([q1, p1]).ravel(); x2 = np.vstack([q2, p2]).ravel(); x0 = x.ravel()
    ll_basic = loglik(g, nm, q2, p2)
    c = (it - 1) % Q
    V[c] = x2 - x1; U[c] = x1 - x0
    m = min(it, Q)
    Uc, Vc = U[:m].T, V[:m].T
    xt = x1 - Vc @ (np.linalg.inv(Uc.T @ (Uc - Vc)) @ (Uc.T @ (x0 - x1)))
    xt = xt.reshape(x.shape)
    pt = project_p(xt[I:])
    qt = np.array([project_q(r) for r in xt[:I]])
    ll_qn = loglik(g, nm, qt, pt)
    if ll_prev < ll_qn:
        xn, ll_new = np.vstack([qt, pt]), ll_qn
    else:
        xn, ll_new = np.vstack([q2, p2]), ll_basic
    return xn, dict(ll_prev=ll_prev, ll_basic=ll_basic, ll_qn=ll_qn, ll_new=ll_new,
                    reldiff=abs((ll_new - ll_prev) / ll_prev))


def init_x(I, J, K, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((I + J, K))
    x[:I] /= x[:I].sum(1, keepdims=True)
    return x


def main():
    for name, (I, J, K, seed) in {"small_k3": (37, 53, 3, 11), "small_k5": (41, 64, 5, 12)}.items():
        bed, codes = make_cohort(I, J, K, seed)
        g, nm = decode(bed, I)
        x = init_x(I, J, K, seed + 100)
        q, p = x[:I], x[I:]
        # one EM step first so q, p are in the interior
        q_em, p_em = em_q(g, nm, q, p), em_p(g, nm, q, p)
        ll_em = loglik(g, nm, q_em, p_em)
        Hq, zq = grad_hess_q(g, nm, q_em, p_em)
        Hp, zp = grad_hess_p(g, nm, q_em, p_em)
        q1, stq = update_q(g, nm, q_em, p_em)
        p1, stp = update_p(g, nm, q1, p_em)
        xe = np.vstack([q_em, p_em])
        U = np.zeros((3, xe.size)); V = np.zeros((3, xe.size))
        xs, infos = xe.copy(), []
        llp = ll_em
        for it in range(1, 5):
            xs, info = qn_iteration(g, nm, xs, llp, U, V, it, 3)
            llp = info["ll_new"]
            infos.append([info[k] for k in ("ll_prev", "ll_basic", "ll_qn", "ll_new", "reldiff")])
        np.savez_compressed(
            OUT / f"{name}.npz", I=I, J=J, K=K, bed=bed, x0=x,
            miss_snp=(codes == 1).sum(0).astype(np.int64), miss_ind=(codes == 1).sum(1).astype(np.int64),
            ll_x0=loglik(g, nm, q, p), q_em=q_em, p_em=p_em, ll_em=ll_em,
            XtX_q=Hq, Xtz_q=zq, XtX_p=Hp, Xtz_p=zp, q_sqp=q1, st_q=stq, p_sqp=p1, st_p=stp,
            qn_info=np.array(infos), x_qn4=xs)
        print("wrote", name, "ll_em", ll_em, "after 4 QN", llp)


if __name__ == "__main__":
    main()
