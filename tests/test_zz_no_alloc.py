"""The allocation-free entry point pism_gpu_ssa_nuH_noalloc, through the C-ABI.

It serves callers that cannot call cudaMalloc (hosts with their own device
memory pools, code running under a fixed memory budget, and bindings without
access to the CUDA allocator): its scratch is a fixed device
array inside the library, so it takes only inputs and outputs.  This test
checks it against the handle API's compute_nuH path (pism_gpu_ssa_compute_nuH
+ pism_gpu_ssa_get_field) on two calls in a row — the second call starts from the
first call's nu*H, so the shared scratch is reused — and checks the two L1 norms
against their definition.  The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from pism_b200 import _capi, synthetic as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pism_b200.ssa import SSAFD  # noqa: E402

RTOL = 1e-12   # the tolerance of the other FP64 stage-parity tests


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _norms(nuH, nuH_before, dx, dy):
    """|nuH| and |nuH_before - nuH| as SSAFD::compute_nuH_norm defines them (ghosted L1)."""
    Mx, My = nuH.shape[:2]
    wi = np.ones(Mx)
    wj = np.ones(My)
    wi[[0, -1]] += 1
    wj[[0, -1]] += 1
    w = np.outer(wi, wj)[..., None]
    a = (np.abs(nuH) * w).reshape(-1, 2).sum(0) * dx * dy
    b = (np.abs(nuH_before - nuH) * w).reshape(-1, 2).sum(0) * dx * dy
    return np.hypot(*a), np.hypot(*b)


def _compare_twice(g, c, f, underrelax=1.0, gl_mask=None, vel_scale=3e-5):
    """two calls in a row against the handle API on the same velocities; the second call
    starts from the first call's nu*H, so the shared scratch is reused"""
    lib = _capi.load()
    dev = torch.device("cuda", 0)
    Mx, My = g.Mx, g.My
    s = SSAFD(g, c, device=0)
    extra = {"gl_mask": gl_mask} if gl_mask is not None else {}
    s.set_inputs(**{k: f[k] for k in ("thickness", "surface", "bed", "mask", "tauc", "melange")}, **extra)
    s.compute_hardav_staggered()
    hardness = torch.tensor(s.hardness(), device=dev)
    H = torch.tensor(f["thickness"], device=dev)
    mask = torch.tensor(f["mask"], device=dev)
    tauc = torch.tensor(f["tauc"], device=dev)
    glm = torch.tensor(gl_mask, device=dev) if gl_mask is not None else None
    nuH = torch.zeros((Mx, My, 2), dtype=torch.float64, device=dev)
    beta = torch.empty((Mx, My), dtype=torch.float64, device=dev)
    norms = torch.empty(2, dtype=torch.float64, device=dev)
    cgrid, _z = g.to_c()
    ccfg = c.to_c()
    rng = np.random.default_rng(4)
    reg = c.epsilon_ssa
    for call in range(2):
        vel_np = rng.normal(0, vel_scale, (Mx, My, 2))
        vel = torch.tensor(vel_np, device=dev)
        before = nuH.cpu().numpy()
        rc = lib.pism_gpu_ssa_nuH_noalloc(C.byref(cgrid), C.byref(ccfg), _ptr(vel), _ptr(H), _ptr(hardness),
                                          _ptr(mask), _ptr(tauc), _ptr(glm) if glm is not None else None, reg,
                                          underrelax, _ptr(nuH), _ptr(beta), _ptr(norms), None)
        assert rc == _capi.OK, f"call {call}: status {rc}"
        torch.cuda.synchronize()
        # the existing entry point on the same velocity; its stage call does not under-relax,
        # so the relaxation of SSAFD.cc:1061-1064 is applied to its result here
        s.set_initial_guess(vel_np)
        s.compute_nuH_staggered(reg)
        nuH_ref, beta_ref = s.nuH(), s.beta()
        if underrelax != 1.0:
            nuH_ref = nuH_ref * underrelax + (1.0 - underrelax) * before
        got = nuH.cpu().numpy()
        np.testing.assert_allclose(got, nuH_ref, rtol=RTOL)
        np.testing.assert_allclose(beta.cpu().numpy(), beta_ref, rtol=RTOL)
        n_ref, d_ref = _norms(got, before, g.dx, g.dy)
        n_got, d_got = norms.cpu().numpy()
        assert n_got == pytest.approx(n_ref, rel=RTOL)
        assert d_got == pytest.approx(d_ref, rel=RTOL)
    s.close()


def test_nuH_noalloc_matches_handle_api_twice():
    g, c, f, _ = S.build_synthetic(67, 4000e3 / 66, seed=11)
    _compare_twice(g, c, f)


def test_nuH_noalloc_under_relaxation():
    """Picard strategy 1's under-relaxation, nu*H <- f nu*H + (1 - f) nu*H_old"""
    g, c, f, _ = S.build_synthetic(67, 4000e3 / 66, seed=12)
    _compare_twice(g, c, f, underrelax=c.ssafd_nuH_iter_failure_underrelaxation)


def test_nuH_noalloc_sub_grounding_line():
    """sub_groundingline: the drag of every icy cell scaled by gl_mask (SSAFD.cc:755-759)"""
    g, c, f, _ = S.build_synthetic(67, 4000e3 / 66, seed=13)
    c = c.copy(sub_groundingline=True)
    gl = np.random.default_rng(5).uniform(0.0, 1.0, (g.Mx, g.My))
    _compare_twice(g, c, f, gl_mask=gl)


def test_nuH_noalloc_thin_grid_with_more_tiles_than_blocks():
    """a grid well inside the cell limit whose 32 x 8 tiles outnumber the scratch's blocks
    (200 000 x 3 cells: 25 000 tiles for 16 384 partial sums): the blocks walk the tiles"""
    from pism_b200.config import GridDesc, SSAConfig
    Mx, My = 200_000, 3
    assert Mx * My <= _capi.NOALLOC_MAX_CELLS and ((My + 31) // 32) * ((Mx + 7) // 8) > _capi.NOALLOC_MAX_CELLS // 256
    g = GridDesc(Mx, My, 0.5 * (Mx - 1) * 5e3, 5e3)
    c = SSAConfig(flow_law="isothermal_glen")
    rng = np.random.default_rng(6)
    H = rng.uniform(0, 2000, (Mx, My))
    bed = rng.uniform(-800, 800, (Mx, My))
    f = {"thickness": H, "bed": bed, "surface": bed + H, "mask": rng.choice([0.0, 2.0, 3.0, 4.0], (Mx, My)),
         "tauc": rng.uniform(1e3, 2e5, (Mx, My)), "melange": None}
    _compare_twice(g, c, f)


def test_nuH_noalloc_rejects_grids_beyond_its_scratch():
    from pism_b200.config import GridDesc, SSAConfig
    lib = _capi.load()
    g = GridDesc(2049, 2048, 1e6, 1e6)
    cgrid, _z = g.to_c()
    ccfg = SSAConfig().to_c()
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = _ptr(t)
    rc = lib.pism_gpu_ssa_nuH_noalloc(C.byref(cgrid), C.byref(ccfg), p, p, p, p, p, None, 0.0, 1.0, p, p, p,
                                      None)
    assert rc == _capi.ETOOLARGE
    assert 2049 * 2048 > _capi.NOALLOC_MAX_CELLS
