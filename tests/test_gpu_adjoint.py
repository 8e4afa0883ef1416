"""Gradients of the Lanczos Green function with respect to the ensemble (adjoint of apply_full_L
and of the averages): the device VJP of the averages against float64 torch autograd of the
restated averages, the differentiable apply and the whole chain against central finite
differences, and dG/d(k3, k4) through the linear force dependence."""
import types

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _ens_obj(d, Y=None, rho=None):
    n = d["X"].shape[1]
    return types.SimpleNamespace(T=d["T"], nat=16, m=np.ones(48), w=d["w"], pols=np.eye(48, n), N=len(d["rho"]),
                                 rho=d["rho"] if rho is None else rho, X=d["X"], Y=d["Y"] if Y is None else Y,
                                 symmetries=d["syms"], deg_space=d["blocks"], blocks_ids=d["blocks_ids"],
                                 supercell=(2, 2, 2), nat_uc=2)


def _lanczos(d, Y=None, rho=None):
    from tdscha_b200 import DynamicalLanczos as DL
    L = DL.Lanczos(_ens_obj(d, Y, rho))
    L.init()
    return L


def _sym(rng, nb, n, scale):
    A = rng.standard_normal((nb, n, n)) * scale
    return A + A.transpose(0, 2, 1)


def test_average_vjp_matches_torch_autograd(cuda, rocksalt_l2):
    from oracle import averages_torch as AT
    d = rocksalt_l2
    n = d["X"].shape[1]
    L = _lanczos(d)
    rng = np.random.default_rng(21)
    nb = 2
    R1 = rng.standard_normal((nb, n)) * 1e-2
    Ys = _sym(rng, nb, n, 1e-2)
    fb = rng.standard_normal((nb, n))
    Db = _sym(rng, nb, n, 1.0)
    S = AT.full_symmetries(d["syms"], d["blocks"], n)
    for d4 in (1, 0):
        Yt = torch.tensor(d["Y"], dtype=torch.float64, requires_grad=True)
        rt = torch.tensor(d["rho"], dtype=torch.float64, requires_grad=True)
        Phi = 0
        for k in range(nb):
            f, D = AT.perturb_average(torch.as_tensor(d["X"]), Yt, d["w"], rt, torch.as_tensor(R1[k]), torch.as_tensor(Ys[k]),
                                      d["T"], d4, S)
            Phi = Phi + (torch.as_tensor(fb[k]) * f).sum() + (torch.as_tensor(Db[k]) * D).sum()
        gY, gr = torch.autograd.grad(Phi, (Yt, rt))
        c = lambda a: torch.as_tensor(a, device="cuda").contiguous()   # noqa: E731
        Ybar = torch.empty((L.N, n), dtype=torch.float64, device="cuda")
        rbar = torch.empty(L.N, dtype=torch.float64, device="cuda")
        L.device_ensemble.perturb_average_vjp(c(R1), c(Ys), c(fb), c(Db), Ybar, rbar, apply_d4=d4)
        assert np.abs(Ybar.cpu().numpy() - gY.numpy()).max() <= 1e-10 * np.abs(gY.numpy()).max()
        assert np.abs(rbar.cpu().numpy() - gr.numpy()).max() <= 1e-10 * np.abs(gr.numpy()).max()


@pytest.mark.parametrize("precision,tol", [("bf16x3", 1e-4), ("tf32x3", 2e-5)])
def test_mixed_precision_vjp_matches_fp64(cuda, rocksalt_l2, precision, tol):
    """The averages' VJP with its contractions on the tcgen05 kernel (tdscha_perturb_average_vjp_
    precision_device) against the FP64 VJP (pinned to float64 torch autograd above)."""
    d = rocksalt_l2
    n = d["X"].shape[1]
    L = _lanczos(d)
    rng = np.random.default_rng(22)
    nb = 3
    R1 = rng.standard_normal((nb, n)) * 1e-2
    Ys = _sym(rng, nb, n, 1e-2)
    fb = rng.standard_normal((nb, n))
    Db = _sym(rng, nb, n, 1.0)
    c = lambda a: torch.as_tensor(a, device="cuda").contiguous()   # noqa: E731
    for d4 in (1, 0):
        out = {}
        for prec in ("fp64", precision):
            Ybar = torch.empty((L.N, n), dtype=torch.float64, device="cuda")
            rbar = torch.empty(L.N, dtype=torch.float64, device="cuda")
            L.device_ensemble.perturb_average_vjp(c(R1), c(Ys), c(fb), c(Db), Ybar, rbar, apply_d4=d4, precision=prec)
            out[prec] = (Ybar.cpu().numpy(), rbar.cpu().numpy())
        eY = np.abs(out[precision][0] - out["fp64"][0]).max() / np.abs(out["fp64"][0]).max()
        er = np.abs(out[precision][1] - out["fp64"][1]).max() / np.abs(out["fp64"][1]).max()
        print(f"VJP {precision} d4={d4}: Ybar {eY:.2e} rhobar {er:.2e}")
        assert eY < tol and er < tol


def test_apply_adjoint_matches_finite_differences(cuda, rocksalt_l2):
    from tdscha_b200 import adjoint
    d = rocksalt_l2
    L = _lanczos(d)
    rng = np.random.default_rng(4)
    ln = len(L.psi)
    v = torch.as_tensor(rng.standard_normal((2, ln)) * 1e-2, device="cuda")
    gbar = torch.as_tensor(rng.standard_normal((2, ln)), device="cuda")
    Yt = torch.tensor(d["Y"], device="cuda", requires_grad=True)
    rt = torch.tensor(d["rho"], device="cuda", requires_grad=True)
    out = adjoint.apply_full_L(v, Yt, rt, L, [0, 1])
    gY, gr = torch.autograd.grad((out * gbar).sum(), (Yt, rt))
    dY = rng.standard_normal(d["Y"].shape)
    dr = rng.standard_normal(d["rho"].shape) * 0.1

    def value(Y, rho):
        Lp = _lanczos(d, Y=Y, rho=rho)
        o = torch.empty_like(v)
        Lp.device_ensemble.apply_full_L(v, o, [0, 1], Lp._opts(), "fp64")
        return float((o * gbar).sum())

    hY = 1e-5 * np.abs(d["Y"]).max()
    fdY = (value(d["Y"] + hY * dY, d["rho"]) - value(d["Y"] - hY * dY, d["rho"])) / (2 * hY)
    adY = float((gY.cpu().numpy() * dY).sum())
    assert abs(adY - fdY) <= 1e-6 * abs(fdY)
    hr = 1e-5
    fdr = (value(d["Y"], d["rho"] + hr * dr) - value(d["Y"], d["rho"] - hr * dr)) / (2 * hr)
    adr = float((gr.cpu().numpy() * dr).sum())
    assert abs(adr - fdr) <= 1e-6 * abs(fdr)


def test_green_function_chain_forward_and_gradient(cuda, rocksalt_l2):
    from tdscha_b200 import adjoint
    d = rocksalt_l2
    L = _lanczos(d)
    L.prepare_mode(4)
    w = np.linspace(0.2, 1.2, 16) * float(np.max(d["w"]))
    eta = 0.05 * float(np.max(d["w"]))
    steps = 8
    # forward agrees with the library's chain + continued fraction
    Lr = _lanczos(d)
    Lr.prepare_mode(4)
    Lr.run_FT(steps, verbose=False)
    g_lib = Lr.get_green_function_continued_fraction(w, use_terminator=False, smearing=eta)
    Yt = torch.tensor(d["Y"], device="cuda", requires_grad=True)
    rt = torch.tensor(d["rho"], device="cuda", requires_grad=True)
    G = adjoint.green_function(L, w, eta, steps, Yt, rt, checkpoint_every=3)
    assert np.abs(G.detach().cpu().numpy() - g_lib).max() <= 1e-10 * np.abs(g_lib).max()
    wts = torch.as_tensor(np.random.default_rng(3).standard_normal(len(w)), device="cuda")
    loss = (G.imag * wts).sum()
    gY, gr = torch.autograd.grad(loss, (Yt, rt))
    rng = np.random.default_rng(9)
    dY = rng.standard_normal(d["Y"].shape)
    dr = rng.standard_normal(d["rho"].shape) * 0.1

    def value(Y, rho):
        Lp = _lanczos(d, Y=Y, rho=rho)
        Lp.prepare_mode(4)
        with torch.no_grad():
            Gp = adjoint.green_function(Lp, w, eta, steps, torch.as_tensor(Y, device="cuda"), torch.as_tensor(rho, device="cuda"))
        return float((Gp.imag * wts).sum())

    hY = 1e-5 * np.abs(d["Y"]).max()
    fdY = (value(d["Y"] + hY * dY, d["rho"]) - value(d["Y"] - hY * dY, d["rho"])) / (2 * hY)
    assert abs(float((gY.cpu().numpy() * dY).sum()) - fdY) <= 1e-6 * abs(fdY)
    hr = 1e-5
    fdr = (value(d["Y"], d["rho"] + hr * dr) - value(d["Y"], d["rho"] - hr * dr)) / (2 * hr)
    assert abs(float((gr.cpu().numpy() * dr).sum()) - fdr) <= 1e-6 * abs(fdr)


def test_green_function_gradient_wrt_couplings(cuda):
    from tdscha_b200 import adjoint, rocksalt as RS
    from tdscha_b200 import DynamicalLanczos as DL
    s = RS.build_system(2)
    X, Y3, Y4, rho = RS.sample_force_components(s, 40, seed=5)

    def lanczos(Y):
        ens = RS.SyntheticEnsemble(T=s.T, nat=s.nat, m=s.masses, w=s.w, pols=s.pols, N=len(rho), rho=rho, X=X, Y=Y,
                                   symmetries=s.symmetries, deg_space=s.deg_space, blocks_ids=s.blocks_ids, supercell=(2, 2, 2))
        L = DL.Lanczos(ens)
        L.init()
        L.prepare_mode(2)
        return L

    w = np.linspace(50, 350, 64) / RS.RY_TO_CM
    eta = 20.0 / RS.RY_TO_CM          # broad enough that G is smooth in (k3, k4) at finite-difference steps
    steps = 10
    k3, k4 = s.k3, s.k4
    Yt = torch.tensor(k3 * Y3 + k4 * Y4, device="cuda", requires_grad=True)
    rt = torch.tensor(rho, device="cuda")
    G = adjoint.green_function(lanczos(k3 * Y3 + k4 * Y4), w, eta, steps, Yt, rt)
    (gY,) = torch.autograd.grad(G.imag.sum(), (Yt,))
    d3, d4 = adjoint.force_gradient_to_k(gY.cpu().numpy(), Y3, Y4)

    def value(a, b):
        Y = a * Y3 + b * Y4
        with torch.no_grad():
            return float(adjoint.green_function(lanczos(Y), w, eta, steps, torch.as_tensor(Y, device="cuda"), rt).imag.sum())

    def richardson(f, h):   # central differences at h and h / 2, O(h^4)
        c1 = (f(h) - f(-h)) / (2 * h)
        c2 = (f(h / 2) - f(-h / 2)) / h
        return (4 * c2 - c1) / 3

    fd3 = richardson(lambda t: value(k3 + t, k4), 1e-3 * abs(k3))
    fd4 = richardson(lambda t: value(k3, k4 + t), 1e-3 * abs(k4))
    assert abs(d3 - fd3) <= 1e-6 * abs(fd3), (d3, fd3)
    assert abs(d4 - fd4) <= 1e-6 * abs(fd4), (d4, fd4)


def test_gradient_at_the_differentiation_workload_size(cuda):
    """The adjoint at the size of the differentiation workload (rock-salt 3x3x3, n = 159, N = 5000,
    1296 symmetries; a shorter chain of 12 steps, checkpoint every 5): directional derivatives of
    sum_w Im G(w) along random directions of the forces and weights against Richardson-extrapolated
    central differences."""
    from tdscha_b200 import adjoint, rocksalt as RS
    from tdscha_b200 import DynamicalLanczos as DL
    s = RS.build_system(3)
    X, Y, rho = RS.sample_ensemble(s, 5000, seed=0)

    def lanczos(Yv, rv):
        ens = RS.SyntheticEnsemble(T=s.T, nat=s.nat, m=s.masses, w=s.w, pols=s.pols, N=len(rv), rho=rv, X=X, Y=Yv,
                                   symmetries=s.symmetries, deg_space=s.deg_space, blocks_ids=s.blocks_ids,
                                   supercell=(3, 3, 3))
        L = DL.Lanczos(ens)
        L.init()
        L.prepare_random(seed=RS.CHAIN_SEED, sector="R")
        return L

    w = np.linspace(50, 350, 64) / RS.RY_TO_CM
    eta = 20.0 / RS.RY_TO_CM
    steps = 12
    Yt = torch.tensor(Y, device="cuda", requires_grad=True)
    rt = torch.tensor(rho, device="cuda", requires_grad=True)
    G = adjoint.green_function(lanczos(Y, rho), w, eta, steps, Yt, rt, checkpoint_every=5)
    gY, gr = torch.autograd.grad(G.imag.sum(), (Yt, rt))
    rng = np.random.default_rng(23)
    dY = rng.standard_normal(Y.shape)
    dr = rng.standard_normal(rho.shape) * 0.1

    def value(Yv, rv):
        L = lanczos(Yv, rv)
        with torch.no_grad():
            v = float(adjoint.green_function(L, w, eta, steps, torch.as_tensor(Yv, device="cuda"),
                                             torch.as_tensor(rv, device="cuda")).imag.sum())
        L.device_ensemble.close()
        return v

    def richardson(f, h):   # central differences at h and h / 2, O(h^4)
        c1 = (f(h) - f(-h)) / (2 * h)
        c2 = (f(h / 2) - f(-h / 2)) / h
        return (4 * c2 - c1) / 3

    fdY = richardson(lambda t: value(Y + t * dY, rho), 1e-4 * np.abs(Y).max())
    adY = float((gY.cpu().numpy() * dY).sum())
    # the weights enter G(w) through the chain, whose rounding makes the difference quotients
    # themselves uncertain at the 1e-6 level here: the bound adds the spread of two step sizes
    fdr = richardson(lambda t: value(Y, rho + t * dr), 1e-3)
    fdr2 = richardson(lambda t: value(Y, rho + t * dr), 2e-3)
    adr = float((gr.cpu().numpy() * dr).sum())
    print(f"3x3x3 N=5000 gradient: Y {adY:.10e} vs FD {fdY:.10e}; rho {adr:.10e} vs FD {fdr:.10e} "
          f"(step 2h: {fdr2:.10e})")
    assert abs(adY - fdY) <= 1e-6 * abs(fdY)
    assert abs(adr - fdr) <= 1e-6 * abs(fdr) + 2 * abs(fdr - fdr2)
