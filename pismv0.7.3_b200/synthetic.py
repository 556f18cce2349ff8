"""Seeded synthetic ice-sheet geometries for the 801 x 801 benchmark and the ensembles.

No public dataset backs the SSA benchmark, so the inputs are generated here from
documented, seeded distributions (numpy PCG64):

* bed: a Gaussian random field (spectral filter with Gaussian covariance,
  correlation length ``corr_len``), standardised to mean -300 m / std 800 m, then
  blended to -3000 m within ``border`` of the domain edges so that the periodic
  wrap of the grid only couples ice-free deep ocean;
* ice surface: the sum of 6 truncated Gaussian domes
  ``A_k * max(exp(-r^2 / (2 s_k^2)) - e^-2, 0) / (1 - e^-2)`` (zero beyond 2 s_k),
  amplitudes A_k ~ U[600, 1200] m, widths s_k ~ U[0.08, 0.12] * domain width,
  centres ~ U[0.3, 0.7] * domain width; thickness = min(s - b, s / alpha)
  (grounded where s - b is the smaller, afloat otherwise; alpha = 1 - rho_i/rho_w),
  clipped to [0, 4000] m.  Taking the domes as the thickness itself would put an
  800 m-rough bed under the ice surface: grounded driving stress would then exceed
  the 50 kPa yield stress on most of the sheet and the plastic-till SSA would have
  no bounded solution;
* mask and surface: GeometryCalculator::compute (src/base/util/Mask.hh:82-118) at
  sea level 0 with rho_ice 910 and rho_sw 1028;
* tau_c: lognormal, median ``tauc_median`` (50 kPa), sigma 1.0, spatially
  correlated over 50 km (a second Gaussian random field);
* hardness: uniform ice at ``temperature_c`` (-10 C).  At exactly the
  Paterson-Budd critical temperature 263.15 K the warm branch applies
  (flowlaws.cc:90-95), so the run uses isothermal Glen with that softness.
"""
from __future__ import annotations

import math

import numpy as np

from .config import SSAConfig, GridDesc


def _grf(rng, M, dx, corr_len):
    """Gaussian random field with covariance exp(-r^2 / corr_len^2), unit variance."""
    k = 2 * np.pi * np.fft.fftfreq(M, d=dx)
    KX, KY = np.meshgrid(k, k, indexing="ij")
    spec = np.exp(-(KX ** 2 + KY ** 2) * corr_len ** 2 / 8.0)   # sqrt of the PSD
    noise = rng.standard_normal((M, M))
    f = np.real(np.fft.ifft2(np.fft.fft2(noise) * spec))
    return (f - f.mean()) / f.std()


def paterson_budd_softness(T_pa: float, cfg: SSAConfig) -> float:
    """FlowLaw::softness_parameter_paterson_budd (flowlaws.cc:90-95)."""
    R = cfg.ideal_gas_constant
    if T_pa < cfg.Paterson_Budd_critical_temperature:
        return cfg.Paterson_Budd_A_cold * math.exp(-cfg.Paterson_Budd_Q_cold / (R * T_pa))
    return cfg.Paterson_Budd_A_warm * math.exp(-cfg.Paterson_Budd_Q_warm / (R * T_pa))


def geometry(cfg: SSAConfig, bed, thickness, sea_level=0.0):
    """GeometryCalculator::compute (Mask.hh:82-118)."""
    alpha = 1.0 - cfg.ice_density / cfg.sea_water_density
    hgrounded = bed + thickness
    hfloating = sea_level + alpha * thickness
    is_floating = hfloating > hgrounded + cfg.mask_is_floating_thickness_standard
    ice_free = thickness < cfg.mask_icefree_thickness_standard
    surface = np.where(is_floating, hfloating, hgrounded)
    mask = np.where(is_floating, np.where(ice_free, 4.0, 3.0), np.where(ice_free, 0.0, 2.0))
    return mask, surface


def build_synthetic(M: int = 801, dx: float = 5.0e3, seed: int = 0, temperature_c: float = -10.0,
                    tauc_median: float = 50.0e3, corr_len: float = 100.0e3, border: float = 150.0e3,
                    cfg: SSAConfig | None = None):
    """Config-2 style synthetic case on an M x M grid of spacing dx."""
    rng = np.random.Generator(np.random.PCG64(seed))
    L = (M - 1) * dx
    grid = GridDesc.shallow(M, M, L / 2, L / 2, periodicity=0)
    cfg = (cfg or SSAConfig()).copy()
    cfg.flow_law = "isothermal_glen"
    cfg.ice_softness = paterson_budd_softness(273.15 + temperature_c, cfg)
    cfg.do_pseudo_plastic_till = False
    cfg.calving_front_stress_boundary_condition = False
    cfg.ssafd_relative_convergence = 1e-4
    cfg.ksp_rtol = 1e-8

    bed = -300.0 + 800.0 * _grf(rng, M, dx, corr_len)
    x = np.arange(M) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    dist = np.minimum(np.minimum(X, L - X), np.minimum(Y, L - Y))
    taper = np.clip(1.0 - dist / border, 0.0, 1.0)
    bed = bed * (1.0 - taper) + (-3000.0) * taper

    srf = np.zeros((M, M))
    cut = math.exp(-2.0)
    domes = []
    for _ in range(6):
        A = rng.uniform(600.0, 1200.0)
        s = rng.uniform(0.08, 0.12) * L
        cx, cy = rng.uniform(0.3, 0.7, size=2) * L
        r2 = (X - cx) ** 2 + (Y - cy) ** 2
        srf += A * np.maximum(np.exp(-r2 / (2 * s * s)) - cut, 0.0) / (1.0 - cut)
        domes.append((A, s, cx, cy))
    alpha = 1.0 - cfg.ice_density / cfg.sea_water_density
    H = np.clip(np.minimum(srf - bed, srf / alpha), 0.0, 4000.0)
    mask, surface = geometry(cfg, bed, H, cfg.sea_level)
    tauc = tauc_median * np.exp(1.0 * _grf(rng, M, dx, 50.0e3))
    fields = {
        "thickness": H, "surface": surface, "bed": bed, "mask": mask, "tauc": tauc,
        "bc_mask": None, "bc_values": None, "melange": np.zeros((M, M)),
    }
    meta = {"seed": seed, "M": M, "dx": dx, "domes": domes, "temperature_c": temperature_c,
            "tauc_median": tauc_median, "corr_len": corr_len, "border": border}
    return grid, cfg, fields, meta
