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


def ref_params():
    """rf_ext_params of the reference-constants mode (the other bond fields are ignored)."""
    x = rfdem.ExtParams()
    x.ref_mode = 1
    x.kn, x.ks, x.bond_lambda, x.gap_frac, x.weibull_m, x.sigma_c, x.tau_c = 1.0, 1.0, 1.0, 0.1, 5.0, 1.0, 1.0
    return x


def ref_mode_case(kind, d, h, seed, **kw):
    """A reference-model lattice specimen (make_test, granite) with what the extended
    model's reference-constants mode needs: (task, R float32, R float64, radius, params)."""
    t, R = rfdem.make_test(kind, d, h, seed=seed, **kw)
    N = int(t.N)
    return t, R, R.astype(np.float64), np.full(N, float(t.Po.p_r)), ref_params()


def pair_counts(R, N, K, IL, ILtype, radius):
    """(bond slots, type-0 slots whose pair overlaps) of a state in the reference layout."""
    P = np.asarray(R, np.float64).reshape(3, N)
    rows = np.asarray(IL, np.uint64).reshape(N, K)
    ty = np.asarray(ILtype).reshape(N, K)
    i, k = np.nonzero(rows < np.uint64(N))
    j = rows[i, k].astype(np.int64)
    d = np.sqrt(((P[:, j] - P[:, i]) ** 2).sum(0))
    r = np.broadcast_to(np.asarray(radius, np.float64), (N,))
    bonds = int((ty[i, k] == 1).sum())
    contacts = int(((ty[i, k] == 0) & (d < r[i] + r[j])).sum())
    return bonds, contacts
