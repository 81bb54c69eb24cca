"""GPU checks of the adjoints of H*y and H\\y (hmatrix.autodiff) on the
differentiation configuration scaled to a size the dense FP64 reference handles:
Gaussian kernel exp(-(x-y)^2/(2 l^2)) + sigma2 I, l = 0.7, sigma2 = 1e-2, points
on [0,10], MaxRank 24, ACA tolerance 1e-10, loss L = b'(H\\b) + |H b|^2.

* the derivative kernels: H-matrices of dK/dp against the dense derivative;
* gradients against the dense FP64 gradient (tolerance 1e-5: the H-matrix is
  within 1e-10 of K, amplified by cond(H) ~ 1e4 in the solves);
* gradients in b, l and sigma2 against central finite differences (step
  1e-6 for l and sigma2) of the H-path loss itself: b enters quadratically,
  sigma2 only shifts the diagonal leaves, and the H-matrices at l +- h are
  built on the structure and aca2 pivots of H (new_like), so their factors
  move smoothly with l: 1e-6.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 4096


def prm(hm, ell=0.7, sigma2=1e-2, kernel=None, keep=False):
    return hm.Params(Geom=np.linspace(0, 10, N), Kernel=kernel or hm.Gauss(ell), MaxBlock=512, MinBlock=64,
                     MaxRank=24, ConsMethod="aca2", εComp=1e-10, Tree="bisect", Shift=sigma2, KeepPivots=keep)


@pytest.mark.parametrize("kind", ["Gauss", "Cauchy", "InvQuad"])
def test_derivative_kernels_vs_dense(kind):
    import hmatrix as hm
    k = getattr(hm, kind)(0.7 if kind != "InvQuad" else 2.0)
    c, H = hm.NewHmat(prm(hm, kernel=k.dp(), sigma2=0.0))
    D = hm.FullMat(k.dp(), c.X, c.X)
    # the derivative kernel is the derivative of the kernel (central difference)
    h = 1e-6
    kp, km = type(k)(k.p + h), type(k)(k.p - h)
    Dfd = (hm.FullMat(kp, c.X, c.X) - hm.FullMat(km, c.X, c.X)) / (2 * h)
    assert np.abs(Dfd - D).max() <= 1e-7 * np.abs(D).max()
    x = np.random.default_rng(1).standard_normal(N)
    assert np.linalg.norm(H * x - D @ x) <= 1e-8 * np.linalg.norm(D @ x)


def _dense_loss_grad(K, dK, s2, b):
    Hd = K + s2 * np.eye(len(b))
    x = np.linalg.solve(Hd, b)
    hb = Hd @ b
    L = b @ x + hb @ hb
    gb = x + np.linalg.solve(Hd.T, b) + 2 * Hd.T @ hb
    gl = -x @ dK @ x + 2 * hb @ dK @ b
    gs = -x @ x + 2 * hb @ b
    return L, gb, gl, gs


def test_gradients_vs_dense_and_fd():
    import torch
    import hmatrix as hm
    from hmatrix.autodiff import KernelOperator
    P = prm(hm, keep=True)
    op = KernelOperator(P, refine_tol=1e-13)
    b0 = np.random.default_rng(4).standard_normal(N)
    b = torch.tensor(b0, device="cuda", requires_grad=True)
    L = torch.dot(b, op.solve(b)) + torch.sum(op.matvec(b) ** 2)
    L.backward()
    gb, gl, gs = b.grad.cpu().numpy(), float(op.p.grad), float(op.sigma2.grad)

    K = hm.FullMat(hm.Gauss(0.7), op.c.X, op.c.X)
    dK = hm.FullMat(hm.GaussDP(0.7), op.c.X, op.c.X)
    Ld, gbd, gld, gsd = _dense_loss_grad(K, dK, 1e-2, b0)
    assert abs(float(L.detach()) - Ld) <= 1e-6 * abs(Ld)
    assert np.linalg.norm(gb - gbd) <= 1e-5 * np.linalg.norm(gbd)
    assert abs(gl - gld) <= 1e-5 * abs(gld)
    assert abs(gs - gsd) <= 1e-5 * abs(gsd)

    # finite differences of the H-path loss
    def loss(op_, bb):
        with torch.no_grad():
            t = torch.tensor(bb, device="cuda")
            return float(torch.dot(t, op_.solve(t)) + torch.sum(op_.matvec(t) ** 2))
    d = np.random.default_rng(5).standard_normal(N)
    h = 1e-3
    fd_b = (loss(op, b0 + h * d) - loss(op, b0 - h * d)) / (2 * h)
    assert abs(fd_b - gb @ d) <= 1e-6 * abs(gb @ d)
    hs = 1e-6
    opp = KernelOperator(prm(hm, sigma2=1e-2 + hs), cluster=op.c, refine_tol=1e-13)
    opm = KernelOperator(prm(hm, sigma2=1e-2 - hs), cluster=op.c, refine_tol=1e-13)
    fd_s = (loss(opp, b0) - loss(opm, b0)) / (2 * hs)
    assert abs(fd_s - gs) <= 1e-6 * abs(gs)
    # l: H at l +- h on H's structure and pivots
    hl = 1e-6
    olp = KernelOperator(prm(hm, ell=0.7 + hl), like=op, refine_tol=1e-13)
    olm = KernelOperator(prm(hm, ell=0.7 - hl), like=op, refine_tol=1e-13)
    fd_l = (loss(olp, b0) - loss(olm, b0)) / (2 * hl)
    assert abs(fd_l - gl) <= 1e-6 * abs(gl), (fd_l, gl)


def test_new_like_replays_the_structure():
    # the same kernel on the same pivots reproduces H bit for bit; another
    # parameter keeps the partition and ranks and stays an accurate H-matrix
    import hmatrix as hm
    c, H = hm.NewHmat(prm(hm, keep=True))
    H2 = hm.new_like(H, prm(hm))
    assert np.array_equal(H.leaves(), H2.leaves())
    x = np.random.default_rng(8).standard_normal(N)
    assert np.array_equal(H * x, H2 * x)
    H3 = hm.new_like(H, prm(hm, ell=0.71, sigma2=0.02))
    assert np.array_equal(H.leaves()[:, :5], H3.leaves()[:, :5])
    K3 = hm.FullMat(hm.Gauss(0.71), c.X, c.X) + 0.02 * np.eye(N)
    assert np.linalg.norm(H3 * x - K3 @ x) <= 1e-8 * np.linalg.norm(K3 @ x)
    bad = prm(hm)
    bad.MaxRank = 12                      # only the kernel and the shift may change
    with pytest.raises(hm.HmError):
        hm.new_like(H3, bad)


def test_matvec_and_solve_adjoints_multi_column():
    # <g, H y> = <H' g, y> and <g, H\\y> = <H'\\g, y> through autograd
    import torch
    import hmatrix as hm
    from hmatrix.autodiff import KernelOperator
    op = KernelOperator(prm(hm, kernel=hm.Cauchy(1.3), sigma2=1.0))
    rng = np.random.default_rng(6)
    Y = torch.tensor(rng.standard_normal((N, 3)), device="cuda", requires_grad=True)
    G = torch.tensor(rng.standard_normal((N, 3)), device="cuda")
    torch.sum(G * op.matvec(Y)).backward()
    ref = op.H.matvec(G.contiguous(), trans=True)
    assert torch.allclose(Y.grad, ref, rtol=1e-13, atol=1e-12)
    Y.grad = None
    torch.sum(G * op.solve(Y)).backward()
    X = torch.linalg.solve(torch.tensor(op.H.to_dense(), device="cuda").T, G)
    assert torch.linalg.norm(Y.grad - X) <= 1e-8 * torch.linalg.norm(X)
