"""Sample-versus-pdf histogram tests (chi-square) of the oracle's sampling routines: each
routine's draws must follow the density it reports.  The device's routines equal these
draw for draw on the same uniforms (tests/test_gpu_parity.py: material sampling, medium and
phase against the reference's golden draws, which the oracle also meets, and the
Henyey-Greenstein sampler against the oracle), so the histograms hold for the device too.

Routines: Lambertian::BSDFSampling (src/Kernel/bsdf.cpp:43-69, through Matte),
Phong::BSDFSampling (src/Kernel/bsdf.cpp:127-170, through Glossy with kd = 0),
Isotropic::IsotropicSampling (src/Kernel/phase.cpp:40-54), the Henyey-Greenstein sampler (not
in the reference) and HomogeneousVolume::DistanceSampling
(src/Volume/homogeneousvolume.cpp:168-215)."""
import math

import numpy as np
import pytest
from scipy import stats

import oraclelib as O
from rumi_b200.scene import Matte, Glossy

N_DRAWS = 400_000
P_MIN = 1e-4


def _uniforms(n, k, seed):
    return O.f32(np.random.default_rng(seed).random((n, k), dtype=np.float32))


def _frame(a):
    a = np.asarray(a, np.float64)
    a = a / np.linalg.norm(a)
    t = np.array([1.0, 0.0, 0.0]) if abs(a[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    t1 = np.cross(a, t)
    t1 /= np.linalg.norm(t1)
    return a, t1, np.cross(a, t1)


def _chi2_sphere(dirs, axis, pdf, n_theta=16, n_phi=32, gauss=16, sub=4):
    """Chi-square of unit vectors `dirs` against the solid-angle density pdf(w: (m, 3)) in
    (cos theta, phi) bins about `axis`; bins expecting fewer than 5 draws are pooled.
    Bin probabilities: Gauss-Legendre in cos theta (peaked lobes), midpoints in phi.
    Returns (p-value, total probability the density puts on the sphere)."""
    a, t1, t2 = _frame(axis)
    d = dirs.astype(np.float64)
    ct = np.clip(d @ a, -1.0, 1.0)
    ph = np.arctan2(d @ t2, d @ t1)
    it = np.minimum(((ct + 1.0) * 0.5 * n_theta).astype(int), n_theta - 1)
    ip = np.minimum(((ph + np.pi) / (2 * np.pi) * n_phi).astype(int), n_phi - 1)
    obs = np.bincount(it * n_phi + ip, minlength=n_theta * n_phi).astype(np.float64)
    # expected: d omega = d cos(theta) d phi
    x, wx = np.polynomial.legendre.leggauss(gauss)
    h = 2.0 / n_theta
    gc = (-1.0 + h * (np.arange(n_theta)[:, None] + 0.5 + 0.5 * x[None, :])).reshape(-1)
    wc = np.tile(wx * (0.5 * h), n_theta)
    gp = -np.pi + (np.arange(n_phi * sub) + 0.5) * (2 * np.pi / (n_phi * sub))
    C, Ph = np.meshgrid(gc, gp, indexing="ij")
    S = np.sqrt(np.maximum(0.0, 1.0 - C ** 2))
    w = (C[..., None] * a + (S * np.cos(Ph))[..., None] * t1 + (S * np.sin(Ph))[..., None] * t2).reshape(-1, 3)
    dens = pdf(w).reshape(C.shape) * wc[:, None] * (2 * np.pi / (n_phi * sub))
    prob = dens.reshape(n_theta, gauss, n_phi, sub).sum(axis=(1, 3)).reshape(-1)
    exp = prob * len(d)
    return _chi2(obs, exp), float(prob.sum())


def _chi2(obs, exp):
    small = exp < 5.0
    o = np.append(obs[~small], obs[small].sum())
    e = np.append(exp[~small], exp[small].sum())
    if e[-1] == 0.0:
        assert o[-1] == 0.0, "draws where the density is zero"
        o, e = o[:-1], e[:-1]
    e = e * (o.sum() / e.sum())  # compare shapes; normalisation is checked separately
    chi = float(((o - e) ** 2 / e).sum())
    return float(stats.chi2.sf(chi, len(o) - 1))


def _material_draws(m, wo, n, seed):
    ms = O.material_struct(m)
    u = _uniforms(N_DRAWS, 3, seed)
    out = np.zeros((N_DRAWS, 9), np.float32)
    O.lib().orc_material_sample_n(O.C.byref(ms), O.P(O.f32(wo)), O.P(O.f32(n)), N_DRAWS, O.P(u), O.P(out))
    return out


def _unit(v):
    v = np.asarray(v, np.float64)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("n", [(0.0, 0.0, 1.0), (0.3, 0.8, -0.52), (0.0, -1.0, 0.0)])
def test_lambertian_draws_follow_cosine_over_pi(n):
    n = _unit(n)
    wo = _unit(n + np.array([0.2, -0.1, 0.3]))
    out = _material_draws(Matte(1.0, (1, 1, 1)), wo, n, seed=11)
    wi = out[:, :3]
    assert np.all(np.abs(np.linalg.norm(wi, axis=1) - 1.0) < 1e-5)
    p, mass = _chi2_sphere(wi, n, lambda w: np.maximum(w @ n, 0.0) / np.pi)
    assert p > P_MIN, p
    assert abs(mass - 1.0) < 1e-3
    # the pdf the routine reports is the density it samples from
    c = np.maximum(wi.astype(np.float64) @ n, 1e-4)
    np.testing.assert_allclose(out[:, 8], c / np.pi, rtol=1e-4, atol=1e-6)


@pytest.mark.parametrize("e", [5.0, 20.0, 100.0])
def test_phong_lobe_draws_follow_the_reported_density_at_normal_incidence(e):
    """wo along n: the lobe axis is n and no draw falls below the horizon, so the draws
    must follow (e + 1) / (2 pi) cos^e(alpha) exactly."""
    n = _unit((0.1, 0.2, 0.97))
    out = _material_draws(Glossy(0.0, 1.0, e, (1, 1, 1)), n, n, seed=int(e))
    wi = out[:, :3]
    dens = lambda w: (e + 1.0) / (2 * np.pi) * np.maximum(w @ n, 0.0) ** e
    p, mass = _chi2_sphere(wi, n, dens, n_theta=64 if e > 20 else 16)
    assert p > P_MIN, p
    assert abs(mass - 1.0) < 2e-3
    ca = np.clip(wi.astype(np.float64) @ n, 0.0, 1.0) ** e
    ref = (e + 1.0) / (2 * np.pi) * np.maximum(ca, 1e-4)
    np.testing.assert_allclose(out[:, 8], ref, rtol=2e-4 * max(1.0, e / 10.0))


def test_phong_lobe_angle_at_oblique_incidence():
    """Oblique wo: draws below the horizon are mirrored about the lobe axis (bsdf.cpp:
    147-167), which keeps the angle to the axis, so cos(alpha) follows (e + 1) c^e on [0, 1]."""
    e = 30.0
    n = np.array([0.0, 0.0, 1.0])
    wo = _unit((0.8, 0.0, 0.6))
    v = -wo + 2.0 * (wo @ n) * n
    out = _material_draws(Glossy(0.0, 1.0, e, (1, 1, 1)), wo, n, seed=5)
    ca = np.clip(out[:, :3].astype(np.float64) @ v, 0.0, 1.0)
    assert np.all(out[:, :3].astype(np.float64) @ n >= -1e-6)  # nothing leaves below the surface
    edges = np.linspace(0.0, 1.0, 41) ** (1.0 / 4.0)
    obs = np.histogram(ca, edges)[0].astype(np.float64)
    exp = np.diff(edges ** (e + 1.0)) * len(ca)
    assert _chi2(obs, exp) > P_MIN


@pytest.mark.parametrize("g", [0.0, 0.35, 0.7, -0.5, 0.95])
def test_phase_draws_follow_their_density(g):
    """Isotropic (g = 0, 1/(4 pi)) and Henyey-Greenstein: the draws against the oracle's own
    pdf evaluation (orc_hg_eval), and that pdf integrates to one over the sphere."""
    d = _unit((0.3, -0.4, 0.87))
    u = _uniforms(N_DRAWS, 2, seed=int(1000 * (g + 1)))
    out = np.zeros((N_DRAWS, 4), np.float32)
    O.lib().orc_phase_sample_n(O.P(O.f32(d)), g, N_DRAWS, O.P(u), O.P(out))
    wi = out[:, :3]
    if g == 0.0:
        dens = lambda w: np.full(len(w), 1.0 / (4 * np.pi))
    else:
        hg = np.vectorize(lambda c: O.lib().orc_hg_eval(float(c), g))
        dens = lambda w: hg(np.clip(w @ d, -1.0, 1.0))
    # the phase about the incoming direction d: the isotropic sampler works about -wo = d
    p, mass = _chi2_sphere(wi, d, dens, n_theta=64 if abs(g) > 0.9 else 16, n_phi=16)
    assert p > P_MIN, p
    assert abs(mass - 1.0) < 2e-3
    if g != 0.0:
        np.testing.assert_allclose(out[:, 3], dens(wi.astype(np.float64)), rtol=1e-3)


@pytest.mark.parametrize("sigma_s,sigma_a,smax", [((0.4, 0.3, 0.2), (0.05, 0.1, 0.02), 3.0),
                                                  ((0.4, 0.4, 0.4), (0.05, 0.05, 0.05), 1.5),
                                                  ((2.0, 1.0, 0.5), (0.5, 0.2, 0.1), 10.0)])
def test_free_flight_distances_follow_the_averaged_extinction(sigma_s, sigma_a, smax):
    """DistanceSampling draws a distance with the channel-averaged extinction sigma: it
    leaves the medium with probability exp(-sigma smax), is absorbed at an interaction
    with probability avg(sigma_a / sigma_t), and otherwise scatters at a distance with
    density proportional to sigma exp(-sigma s) on [0, smax]."""
    ss, sa = np.array(sigma_s, np.float64), np.array(sigma_a, np.float64)
    st = ss + sa
    sig = st.mean()
    absorb = (sa / st).mean()
    u = _uniforms(N_DRAWS, 2, seed=int(smax * 10))
    out = np.zeros((N_DRAWS, 9), np.float32)
    O.lib().orc_distance_sample_n(O.P(O.f32(sigma_s)), O.P(O.f32(sigma_a)), smax, N_DRAWS, O.P(u), O.P(out))
    oc = out[:, 0].astype(int)
    n = len(oc)
    p_pass = math.exp(-sig * smax)
    frac = np.mean(oc == 0)
    assert abs(frac - p_pass) < 4.0 * math.sqrt(p_pass * (1 - p_pass) / n) + 1e-4, (frac, p_pass)
    inter = oc != 0
    fa = np.mean(oc[inter] == 2)
    assert abs(fa - absorb) < 4.0 * math.sqrt(absorb * (1 - absorb) / inter.sum()), (fa, absorb)
    s = out[oc == 1, 1].astype(np.float64)
    assert s.min() >= 1e-4 and s.max() <= smax
    edges = np.linspace(0.0, smax, 33)
    obs = np.histogram(s, edges)[0].astype(np.float64)
    exp = -np.diff(np.exp(-sig * edges))
    assert _chi2(obs, exp * len(s)) > P_MIN
    if np.all(st == st[0]):
        # a grey medium: the per-channel pdf the routine reports is the density it samples
        tau_pdf = out[oc == 1, 5:8].astype(np.float64)
        np.testing.assert_allclose(tau_pdf[:, 0], sig * np.exp(-sig * s), rtol=1e-4)
