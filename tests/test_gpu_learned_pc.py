"""The learned preconditioner correction of flexible GMRES, through the C-ABI: the network
input it builds for a residual against its definition, the solve with a caller's right-hand
side against a direct solve, and FGMRES with the correction attached meeting the same FP64
tolerance (and giving the same answer) as without it."""
import os

import numpy as np
import pytest

from pism_b200 import learned as L, synthetic as S
from oracle import ssafd_oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD  # noqa: E402

NAMES = ("thickness", "surface", "bed", "mask", "tauc", "melange")


def _state(M, seed, picard_rtol=1e-2):
    """a handle at a Picard iterate of a synthetic sheet (FP64 FGMRES + multigrid)"""
    g, c, f, _ = S.build_synthetic(M, 4000e3 / (M - 1), seed=seed)
    c = L.pc_config(c).copy(ssafd_relative_convergence=picard_rtol, ksp_rtol=1e-8)
    s = SSAFD(g, c)
    s.set_inputs(**{k: f[k] for k in NAMES})
    s.solve()
    return g, c, f, s


def _dinv_blocks(A, Mx, My):
    """the inverse 2 x 2 diagonal blocks of the assembled matrix, [Mx, My, 2, 2]"""
    d = A.diagonal()
    off_up = A.diagonal(1)[0::2]    # (2k, 2k+1)
    off_lo = A.diagonal(-1)[0::2]   # (2k+1, 2k)
    blk = np.zeros((Mx * My, 2, 2))
    blk[:, 0, 0], blk[:, 1, 1] = d[0::2], d[1::2]
    blk[:, 0, 1], blk[:, 1, 0] = off_up, off_lo
    return np.linalg.inv(blk).reshape(Mx, My, 2, 2)


@pytest.mark.parametrize("stride", [1, 2])
def test_pc_input_matches_its_definition(stride):
    M = 41
    g, c, f, s = _state(M, 3)
    G, Cc, I = O.from_case(g, c, f)
    A = O.assemble_matrix(G, Cc, I, s.nuH(), s.beta())
    r = np.random.default_rng(4).standard_normal((M, M, 2))
    img, rho = L.pc_input(s, torch.tensor(r, device="cuda"), stride)
    img = img.cpu().numpy()
    feats = L.features(s, stride).cpu().numpy()
    np.testing.assert_array_equal(img[..., :6], feats[..., :6])
    sD = np.einsum("ijab,ijb->ija", _dinv_blocks(A, M, M), r)
    hh, ww = img.shape[:2]
    means = np.zeros((hh, ww, 2))
    for I_ in range(-(-M // stride)):
        for J_ in range(-(-M // stride)):
            blk = sD[I_ * stride:(I_ + 1) * stride, J_ * stride:(J_ + 1) * stride]
            means[I_, J_] = blk.reshape(-1, 2).mean(0)
    rho_ref = np.sqrt((means ** 2).sum() / (2 * hh * ww))
    assert float(rho) == pytest.approx(rho_ref, rel=1e-10)
    np.testing.assert_allclose(img[..., 6:], means / rho_ref, rtol=1e-5, atol=1e-6)
    s.close()


def test_linear_solve_with_a_callers_rhs():
    M = 41
    g, c, f, s = _state(M, 5)
    G, Cc, I = O.from_case(g, c, f)
    s.set_config(c.copy(ksp_rtol=1e-12))
    A = O.assemble_matrix(G, Cc, I, s.nuH(), s.beta())
    b = np.random.default_rng(6).standard_normal((M, M, 2)) * 1e3
    x = torch.zeros((M, M, 2), dtype=torch.float64, device="cuda")
    its, res = s.linear_solve_rhs(torch.tensor(b, device="cuda"), x)
    assert res <= 1e-12
    ref = O.linear_solve(A, b.ravel(), None, "direct").reshape(b.shape)
    assert np.linalg.norm(x.cpu().numpy() - ref) <= 1e-8 * np.linalg.norm(ref)
    # the handle's own right-hand side is untouched
    np.testing.assert_array_equal(s.rhs(), s.rhs())
    s.close()


@pytest.mark.parametrize("stride", [1, 2])
def test_fgmres_with_the_correction_meets_the_same_tolerance(stride):
    """Any correction network (here untrained, or the committed weights) leaves the FP64
    residual test in charge: the same tolerance, the same answer to its accuracy."""
    M = 45
    g, c, f, s = _state(M, 7)
    s.set_config(c.copy(ksp_rtol=1e-10))
    hh, ww = L.image_shape(M, M, stride)
    params = np.load(L.PC_WEIGHTS)["params"] if os.path.exists(L.PC_WEIGHTS) else L.init_params(3)
    net = L.UNet(1, hh, ww, params=params)
    x0 = torch.zeros((M, M, 2), dtype=torch.float64, device="cuda")
    its0, res0 = s.linear_solve(x0)
    L.set_learned_pc(s, net, stride)
    x1 = torch.zeros_like(x0)
    its1, res1 = s.linear_solve(x1)
    L.set_learned_pc(s, None, stride)
    assert res0 <= 1e-10 and res1 <= 1e-10
    assert (x1 - x0).norm() <= 1e-7 * x0.norm()
    print(f"FGMRES(30) + multigrid, 45^2, stride {stride}: {its0} iterations, with the correction {its1}")
    s.close()
    net.close()
