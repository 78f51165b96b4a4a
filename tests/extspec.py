"""Specimens of the extended model for the tests: polydisperse radii on a jittered
lattice (CPU, no packing needed) or packed on the GPU."""
import numpy as np

import rfdem


def lattice_ext(kind, d, h, r0=0.5, seed=0xB2000000 + 7, rlo=0.97, jitter=0.02):
    """Jittered-lattice specimen of spacing 2 r0 with radii r0 * U[rlo, 1], centred at the
    origin. Returns (R double planar, radius double)."""
    Rf = rfdem.specimen_positions(kind, seed, r0, d, h, (0.0, 0.0, 0.0), gap_frac=0.0, jitter=jitter)
    N = Rf.size // 3
    rng = np.random.default_rng(seed)
    rad = r0 * (rlo + (1.0 - rlo) * rng.random(N))
    return Rf.astype(np.float64), rad


def stiff_params(seed=0xB2000000 + 9, weibull_m=5.0, sigma_c=None, tau_c=None):
    """Bond constants near the reference granite's (kn = m_E / (2 r_P), ks = m_G / (2 r_P))
    with Weibull strengths around the reference's critical stresses."""
    po = rfdem.granite_potential()
    x = rfdem.ExtParams()
    m_G = 0.5 * po.m_E / (1.0 + po.m_nu)
    x.kn = po.m_E / (2 * po.p_r)
    x.ks = m_G / (2 * po.p_r)
    x.bond_lambda = po.b_r / po.p_r
    x.gap_frac = 0.05
    x.weibull_m = weibull_m
    x.sigma_c = po.m_Ec if sigma_c is None else sigma_c
    x.tau_c = po.m_Gc if tau_c is None else tau_c
    x.seed = seed
    return x


def ext_case(kind, d, h, r0=0.5, seed=0xB2000000 + 7, **kw):
    """(task, R, radius, params) for a lattice specimen with reference-like bonds."""
    R0, rad = lattice_ext(kind, d, h, r0=r0, seed=seed)
    t, R = rfdem.make_test_ext(kind, R0, rad, r0, **kw)
    return t, R, rad, stiff_params()
