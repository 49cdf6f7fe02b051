"""Backward kernels (ocipProximityBackward): gradients of SqrDistance and
CrossCorr_Norm with respect to the source image and the template.

A torch.autograd.Function (test harness only) runs the forward measures and
the backward through the C ABI. Bars:
  * against the long-double CPU adjoint: max error <= 1e-4 of the gradient's
    largest magnitude (the template gradient sums W*H products of random sign,
    so its entries are ~sqrt(W*H) times smaller than the sum of magnitudes;
    the split-BF16 products, good to ~2^-17 each, leave ~1e-5 of the largest
    entry);
  * against FP64 central finite differences of the long-double forward
    (h = 1e-3, 64 seeded coordinates of the image and of the template):
    agreement <= 1e-4 relative to the largest sampled finite difference of
    the same tensor.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

ADJ_TOL = 1e-4
FD_TOL = 1e-4


def blob_pair(H, W, th, tw, seed):
    import bench
    S = bench.blob_field(W, H, nblobs=12, seed=seed)
    rng = np.random.default_rng(seed)
    y, x = int(rng.integers(0, H - th)), int(rng.integers(0, W - tw))
    T = (S[y:y + th, x:x + tw] + rng.normal(0, 0.02, (th, tw))).astype(np.float32)
    return S, T


def backward(ocip, S, T, G1, G2, out_dtype=np.float32):
    """Gradients from the C ABI; N2 from the tensor forward when G2 is given."""
    Si, Ti = ocip.Image(S), ocip.Image(T)
    keep = [Si, Ti]
    g1 = g2 = n2 = None
    if G1 is not None:
        g1 = ocip.Image(np.ascontiguousarray(G1, np.float32))
        keep.append(g1)
    if G2 is not None:
        N = np.zeros(S.shape, np.float32)
        n2 = ocip.Image(N)
        ocip.check(ocip.cross_corr_norm(Si, Ti, n2), "forward")
        g2 = ocip.Image(np.ascontiguousarray(G2, np.float32))
        keep += [n2, g2]
    dS = np.zeros(S.shape, out_dtype)
    dT = np.zeros(T.shape, out_dtype)
    dSi, dTi = ocip.Image(dS), ocip.Image(dT)
    keep += [dSi, dTi]
    try:
        ocip.check(ocip.proximity_backward(Si, Ti, g1, g2, n2, dSi, dTi), "ocipProximityBackward")
        dSi.read()
        dTi.read()
    finally:
        for k in keep:
            k.release()
    return dS.astype(np.float64), dT.astype(np.float64)


def oracle_adjoint(S, T, G1, G2):
    dS = np.zeros(S.shape)
    dT = np.zeros(T.shape)
    if G1 is not None:
        a, b = O.proximity_backward(0, S, T, G1)
        dS += a
        dT += b
    if G2 is not None:
        a, b = O.proximity_backward(4, S, T, G2)
        dS += a
        dT += b
    return dS, dT


def rel_max(got, ref):
    return float(np.abs(got - ref).max() / np.abs(ref).max())


@pytest.mark.parametrize("th,tw", [(31, 31), (32, 32), (64, 64), (12, 20), (40, 9), (9, 45)])
@pytest.mark.parametrize("which", ["sqr", "ccnorm", "both"])
def test_backward_matches_cpu_adjoint(ocip, ctx, th, tw, which):
    ctx.make_current()
    ctx.set_path(ocip.PATH_TENSOR)
    S, T = blob_pair(150, 280, th, tw, seed=th * 100 + tw)
    rng = np.random.default_rng(7)
    G1 = rng.standard_normal(S.shape).astype(np.float32) if which in ("sqr", "both") else None
    G2 = rng.standard_normal(S.shape).astype(np.float32) if which in ("ccnorm", "both") else None
    dS, dT = backward(ocip, S, T, G1, G2)
    rS, rT = oracle_adjoint(S, T, G1, G2)
    assert rel_max(dS, rS) <= ADJ_TOL, ("dS", rel_max(dS, rS))
    assert rel_max(dT, rT) <= ADJ_TOL, ("dT", rel_max(dT, rT))
    ctx.set_path(ocip.PATH_PLAIN)


def loss(S, T, G1, G2):
    """FP64 (long double) forward of L = sum G1 SqrDistance + sum G2 CrossCorr_Norm."""
    L = 0.0
    if G1 is not None:
        L += float((G1 * O.proximity_exact(0, S, T)).sum())
    if G2 is not None:
        L += float((G2 * O.proximity_exact(4, S, T)).sum())
    return L


def test_backward_finite_differences(ocip, ctx):
    """64 seeded coordinates (32 of the image, 32 of the template), central
    differences with h = 1e-3 on the long-double forward."""
    ctx.make_current()
    ctx.set_path(ocip.PATH_TENSOR)
    S, T = blob_pair(70, 90, 16, 16, seed=3)
    rng = np.random.default_rng(8)
    G1 = rng.standard_normal(S.shape).astype(np.float32)
    G2 = rng.standard_normal(S.shape).astype(np.float32)
    dS, dT = backward(ocip, S, T, G1, G2)
    h = 1e-3
    S64, T64 = S.astype(np.float64), T.astype(np.float64)
    got, fds = {"S": [], "T": []}, {"S": [], "T": []}
    for _ in range(32):
        y, x = int(rng.integers(0, S.shape[0])), int(rng.integers(0, S.shape[1]))
        Sp, Sm = S64.copy(), S64.copy()
        Sp[y, x] += h
        Sm[y, x] -= h
        fds["S"].append((loss(Sp, T64, G1, G2) - loss(Sm, T64, G1, G2)) / (2 * h))
        got["S"].append(dS[y, x])
    for _ in range(32):
        y, x = int(rng.integers(0, T.shape[0])), int(rng.integers(0, T.shape[1]))
        Tp, Tm = T64.copy(), T64.copy()
        Tp[y, x] += h
        Tm[y, x] -= h
        fds["T"].append((loss(S64, Tp, G1, G2) - loss(S64, Tm, G1, G2)) / (2 * h))
        got["T"].append(dT[y, x])
    for k in ("S", "T"):
        fd, g = np.array(fds[k]), np.array(got[k])
        err = np.abs(g - fd).max() / np.abs(fd).max()
        assert err <= FD_TOL, (k, err)
    ctx.set_path(ocip.PATH_PLAIN)


def test_autograd_function_template_refinement(ocip, ctx):
    """The torch.autograd.Function wrapper: gradients flow to both inputs and
    a few gradient steps on the template raise its best CrossCorr_Norm."""
    import torch
    ctx.make_current()
    ctx.set_path(ocip.PATH_TENSOR)

    class Match(torch.autograd.Function):
        @staticmethod
        def forward(c, S, T):
            Sn, Tn = S.detach().cpu().numpy(), T.detach().cpu().numpy()
            sqr = ocip.match("SqrDistance", Sn, Tn)
            ccn = ocip.match("CrossCorr_Norm", Sn, Tn)
            c.save_for_backward(S, T)
            c.ccn = ccn
            return torch.from_numpy(sqr), torch.from_numpy(ccn)

        @staticmethod
        def backward(c, g1, g2):
            S, T = c.saved_tensors
            Sn, Tn = S.detach().cpu().numpy(), T.detach().cpu().numpy()
            Si, Ti = ocip.Image(Sn), ocip.Image(Tn)
            G1 = ocip.Image(np.ascontiguousarray(g1.numpy(), np.float32))
            G2 = ocip.Image(np.ascontiguousarray(g2.numpy(), np.float32))
            N2 = ocip.Image(c.ccn)
            dS = np.zeros(Sn.shape, np.float32)
            dT = np.zeros(Tn.shape, np.float32)
            dSi, dTi = ocip.Image(dS), ocip.Image(dT)
            ocip.check(ocip.proximity_backward(Si, Ti, G1, G2, N2, dSi, dTi), "backward")
            dSi.read()
            dTi.read()
            for k in (Si, Ti, G1, G2, N2, dSi, dTi):
                k.release()
            return torch.from_numpy(dS), torch.from_numpy(dT)

    S, T0 = blob_pair(64, 96, 16, 16, seed=9)
    y, x = 20, 40
    target = S[y:y + 16, x:x + 16].copy()
    S_t = torch.from_numpy(S).requires_grad_(True)
    T_t = torch.from_numpy((target + np.random.default_rng(1).normal(0, 0.1, target.shape))
                           .astype(np.float32)).requires_grad_(True)
    _, ccn = Match.apply(S_t, T_t)
    first = float(ccn[y + 8, x + 8].detach())
    for _ in range(5):
        sqr, ccn = Match.apply(S_t, T_t)
        L = ccn[y + 8, x + 8] - 1e-4 * sqr.mean()
        T_t.grad = None
        S_t.grad = None
        L.backward()
        assert S_t.grad is not None and torch.isfinite(S_t.grad).all()
        with torch.no_grad():
            T_t += 0.05 * T_t.grad / (T_t.grad.abs().max() + 1e-12)
    _, ccn = Match.apply(S_t, T_t)
    assert float(ccn[y + 8, x + 8].detach()) > first
    ctx.set_path(ocip.PATH_PLAIN)


def test_backward_f64_outputs_and_checks(ocip, ctx):
    ctx.make_current()
    S, T = blob_pair(60, 130, 10, 10, seed=4)
    rng = np.random.default_rng(2)
    G1 = rng.standard_normal(S.shape).astype(np.float32)
    dS, dT = backward(ocip, S, T, G1, None, out_dtype=np.float64)
    rS, rT = oracle_adjoint(S, T, G1, None)
    assert rel_max(dS, rS) <= ADJ_TOL and rel_max(dT, rT) <= ADJ_TOL
    Si, Ti = ocip.Image(S), ocip.Image(T)
    Gi = ocip.Image(G1)
    U8 = ocip.Image(rng.integers(0, 255, S.shape, dtype=np.uint8))
    Gs = ocip.Image(np.zeros((10, 10), np.float32))
    try:
        assert ocip.proximity_backward(Si, Ti) == ocip.CL_INVALID_VALUE  # no gradient
        assert ocip.proximity_backward(Si, Ti, None, Gi) == ocip.CL_INVALID_VALUE  # no N2
        assert ocip.proximity_backward(U8, Ti, Gi) == ocip.CL_INVALID_VALUE
        assert ocip.proximity_backward(Si, Ti, Gs) == ocip.CL_INVALID_IMAGE_SIZE
    finally:
        for k in (Si, Ti, Gi, U8, Gs):
            k.release()
