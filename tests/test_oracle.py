"""Pins the CPU FP64 oracle: known-answer tests from published vectors,
numpy, closed-form physics and the reference's own formulas.

The reference ships no tests and its programs cannot be built here (cutil,
GLUT, legacy texture references), so these checks are what the oracle is
trusted on; see also test_golden.py for the reference's stored curves.
"""
import numpy as np
import pytest

from bec_b200 import observables as OBS
from bec_b200._abi import BEC_GS_FIXED_STEPS, BEC_GS_MU, BEC_GS_MU_RESIDUAL, BEC_GS_REFERENCE_E
from bec_b200.configs import slice_2d_32x128, copy_params, rb87_params
from oracle import oracle as O


# ---------------------------------------------------------------- Philox
# Known-answer vectors of Philox4x32-10 published with Random123
# (Salmon et al., SC'11; file kat_vectors).
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,expect", PHILOX_KAT)
def test_philox_known_answers(ctr, key, expect):
    assert tuple(O.philox(ctr, key)) == expect


def test_normals_statistics():
    rng_vals = np.array([O.normals4(7, t, 3, c, 1) for t in range(4) for c in range(5000)]).reshape(-1)
    assert abs(rng_vals.mean()) < 0.02
    assert abs(rng_vals.std() - 1.0) < 0.02
    # kurtosis of a normal is 3
    assert abs(((rng_vals - rng_vals.mean()) ** 4).mean() / rng_vals.var() ** 2 - 3.0) < 0.15


def test_loss_normals_fields_and_statistics():
    """Six normals per Philox draw: the 21-bit fields restated from the draw's words, and the
    moments and mutual independence of the six outputs."""
    seed, traj, step, cell = 0x1234567890AB, 3, 17, 4242
    w = [int(v) for v in O.philox((cell, step, traj, 1), (seed & 0xFFFFFFFF, seed >> 32))]
    bits = w[0] | (w[1] << 32) | (w[2] << 64) | (w[3] << 96)
    f = [(bits >> (21 * k)) & 0x1FFFFF for k in range(6)]
    expect = []
    for k in range(3):
        r = np.sqrt(-2.0 * np.log((f[2 * k] + 0.5) / 2.0 ** 21))
        a = 2.0 * np.pi * f[2 * k + 1] / 2.0 ** 21
        expect += [r * np.cos(a), r * np.sin(a)]
    np.testing.assert_allclose(O.loss_normals6(seed, traj, step, cell), expect, rtol=1e-14, atol=1e-14)
    v = np.array([O.loss_normals6(7, t, 3, c) for t in range(4) for c in range(5000)])
    assert np.all(np.abs(v.mean(axis=0)) < 0.04)
    assert np.all(np.abs(v.std(axis=0) - 1.0) < 0.03)
    assert abs(((v - v.mean()) ** 4).mean() / v.var() ** 2 - 3.0) < 0.15
    corr = np.corrcoef(v.T)
    assert np.max(np.abs(corr - np.eye(6))) < 0.05


# ---------------------------------------------------------------- FFT
@pytest.mark.parametrize("shape", [(64, 8, 8), (128, 16, 16), (128, 1, 32), (16, 4, 2)])
def test_fft_matches_numpy(shape):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = O.fft3d(a, -1)
    np.testing.assert_allclose(f, np.fft.fftn(a), rtol=0, atol=1e-12 * np.abs(f).max())
    b = O.fft3d(a, +1)
    np.testing.assert_allclose(b, np.fft.ifftn(a) * a.size, rtol=0, atol=1e-12 * np.abs(b).max())


# ---------------------------------------------------------------- units
def test_derived_parameters_match_reference_formulas():
    """fillDerivedParameters (wigner.cpp:119-176) at N = 30000."""
    p = rb87_params(N=30000, grid=(16, 16, 128))
    d = O.derive(p)
    hbar, a0 = 1.054571628e-34, 5.2917720859e-11
    w = 2 * np.pi * p.fx
    l_rho = np.sqrt(hbar / (p.m * w))
    assert d.l_rho == pytest.approx(l_rho, rel=1e-15)
    assert d.l_rho == pytest.approx(1.0916e-6, rel=1e-4)
    assert d.t_rho == pytest.approx(1 / w, rel=1e-15)
    assert d.lambda_ == pytest.approx(97.6 / 11.96, rel=1e-15)
    g11 = 4 * np.pi * p.a11 * a0 / l_rho
    mu = (15 * p.N * g11 / (16 * np.pi * d.lambda_ * np.sqrt(2))) ** 0.4
    assert d.mu == pytest.approx(mu, rel=1e-14)
    assert d.mu == pytest.approx(4.682, rel=1e-3)
    assert d.xmax == pytest.approx(1.2 * np.sqrt(2 * mu), rel=1e-14)
    assert d.zmax == pytest.approx(1.2 * d.lambda_ * np.sqrt(2 * mu), rel=1e-14)
    assert d.dx == pytest.approx(2 * d.xmax / 15, rel=1e-14)
    assert d.dkx == pytest.approx(np.pi / d.xmax, rel=1e-15)   # the reference's dk quirk
    assert d.dt_evo == pytest.approx(4e-5 * w, rel=1e-14)
    assert d.l111 == pytest.approx(5.4e-42 / (l_rho ** 6 * w), rel=1e-13)
    assert d.l12 == pytest.approx(1.51e-20 / (l_rho ** 3 * w), rel=1e-13)
    assert d.n_equil_steps == 1            # for (t = 0; t <= 0; ...) runs once


def test_thomas_fermi_normalisation():
    """The TF profile of mu integrates to N (report.tex:63-66) on a fine grid."""
    p = rb87_params(N=30000, grid=(64, 64, 256))
    d = O.derive(p)
    V = O.potential_table(d)
    n = np.maximum(d.mu - V, 0) / d.g11
    assert n.sum() * d.dV == pytest.approx(30000, rel=0.02)


def test_2d_thomas_fermi_normalisation():
    p = rb87_params(N=30000, grid=(256, 1, 1024))
    d = O.derive(p)
    V = O.potential_table(d)
    n = np.maximum(d.mu - V, 0) / d.g11
    assert n.sum() * d.dV == pytest.approx(30000, rel=0.01)


def test_k_table_convention():
    """getK (wigner_kernel.cu:15-21): k = dk i for 2i <= n, else dk (i - n)."""
    p = rb87_params(grid=(8, 8, 64))
    d = O.derive(p)
    k2 = O.k2_table(d).reshape(64, 8, 8)
    kx = np.array([d.dkx * (i if 2 * i <= 8 else i - 8) for i in range(8)])
    assert k2[0, 0, :] == pytest.approx(kx ** 2 / 2, rel=1e-15)
    kz = np.array([d.dkz * (i if 2 * i <= 64 else i - 64) for i in range(64)])
    assert k2[:, 0, 0] == pytest.approx(kz ** 2 / 2, rel=1e-15)


# ---------------------------------------------------------------- ground state
def test_ground_state_converges_and_mu_matches_tf():
    p = rb87_params(N=30000, grid=(16, 16, 128))
    psi, rep = O.ground_state(p, mode=BEC_GS_MU, max_steps=4000, tol=1e-7, check_every=10)
    assert rep.converged == 1
    assert rep.N == pytest.approx(30000, rel=1e-12)
    d = O.derive(p)
    # the kinetic term lowers the density peak; mu stays within 10% of Thomas-Fermi
    assert abs(rep.mu - d.mu) / d.mu < 0.1
    assert rep.residual < 0.05 * rep.mu
    mu2, e2, r2, n2 = O.gs_measures(p, psi)
    assert mu2 == pytest.approx(rep.mu, rel=1e-12)


def test_ground_state_reference_energy_mode_stops():
    p = slice_2d_32x128()
    psi, rep = O.ground_state(p, mode=BEC_GS_REFERENCE_E, max_steps=20000)
    assert rep.converged == 1 and rep.steps < 20000


def test_mu_residual_rule_waits_for_a_stationary_state():
    """From Thomas-Fermi, mu passes through a minimum before it settles, and the mu-only rule
    stops there; the rule that also bounds the fixed-point residual stops on the monotone tail."""
    p = rb87_params(N=30000, grid=(8, 8, 64))
    _, r_mu = O.ground_state(p, mode=BEC_GS_MU, max_steps=20000, tol=1e-6, check_every=20)
    _, r_res = O.ground_state(p, mode=BEC_GS_MU_RESIDUAL, max_steps=20000, tol=1e-6, check_every=20)
    _, r_inf = O.ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=4000)
    assert r_mu.converged and r_res.converged
    assert r_res.steps > r_mu.steps
    assert 0 < r_res.step_residual < 1e-5
    err_mu = abs(r_mu.mu - r_inf.mu) / r_inf.mu
    err_res = abs(r_res.mu - r_inf.mu) / r_inf.mu
    assert err_res < 5e-6 and err_res < err_mu / 2


def test_mu_residual_rule_stops_at_second_check_from_the_fixed_point():
    p = rb87_params(N=30000, grid=(8, 8, 64))
    psi, _ = O.ground_state(p, mode=BEC_GS_FIXED_STEPS, max_steps=4000)
    _, r = O.ground_state(p, mode=BEC_GS_MU_RESIDUAL, max_steps=2000, tol=1e-6, check_every=20, warm_start=psi)
    assert r.converged and r.steps == 40


def test_imaginary_time_lowers_energy():
    p = slice_2d_32x128()
    _, r1 = O.ground_state(p, max_steps=10)
    _, r2 = O.ground_state(p, max_steps=400)
    assert r2.energy < r1.energy
    assert r2.residual < r1.residual


# ---------------------------------------------------------------- evolution
def _small(noise=False, losses=True, ne=1, grid=(8, 8, 64), **kw):
    return rb87_params(N=20000, grid=grid, ne=ne, noise=noise, losses=losses, **kw)


def test_norm_conserved_without_losses():
    p = _small(losses=False)
    gs, _ = O.ground_state(p, max_steps=50)
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution()
    m0 = e.moments()
    e.evolve(50)
    m1 = e.moments()
    assert (m1[1] + m1[2]) == pytest.approx(m0[1] + m0[2], rel=1e-12)


def test_two_body_loss_rate_one_step():
    """Without noise, the nonlinear step multiplies |b|^2 by exp(-l22 n_b dt) (itmax = 1),
    so one step loses l22 dt sum n_b^2 dV to first order (report.tex:317-330)."""
    p = _small(losses=False)
    p.gamma22 = 8.1e-20 * 50
    gs, _ = O.ground_state(p, max_steps=50)
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.pulse(np.pi, 0.0)      # everything into |2>
    # x-space state after the first half kick is what the nonlinear step sees
    d = e.d
    ab = e.get_state(0)
    k2 = O.k2_table(d)
    bk = np.fft.ifftn(ab[1].reshape(d.nvz, d.nvy, d.nvx)).reshape(-1) * np.exp(1j * k2 * d.dt_evo / 2)
    bx = np.fft.fftn(bk.reshape(d.nvz, d.nvy, d.nvx)).reshape(-1)
    nb = np.abs(bx) ** 2
    N0 = nb.sum() * d.dV
    expect = (nb * np.exp(-d.l22 * nb * d.dt_evo)).sum() * d.dV
    e.evolve(1)
    m = e.moments()
    assert m[2] == pytest.approx(expect, rel=1e-12)
    assert N0 - m[2] == pytest.approx(d.l22 * d.dt_evo * (nb ** 2).sum() * d.dV, rel=0.05)


def test_pulses_compose():
    p = _small(losses=False)
    gs, _ = O.ground_state(p, max_steps=20)
    e1, e2 = O.OracleEnsemble(p), O.OracleEnsemble(p)
    e1.init(gs); e2.init(gs)
    e1.pulse(np.pi / 2); e1.pulse(np.pi / 2)
    e2.pulse(np.pi)
    np.testing.assert_allclose(e1.get_state(0), e2.get_state(0), atol=1e-12 * np.abs(gs).max())
    e1.pulse(np.pi, np.pi)   # pi about the opposite axis undoes a pi pulse
    np.testing.assert_allclose(e1.get_state(0)[0], gs, atol=1e-11 * np.abs(gs).max())


def test_visibility_and_projection_closed_forms_match_reference_literal():
    """getVisibility / halfPiRotate / axial projection computed literally (oracle)
    equal the closed forms of bec_b200.observables on the oracle's moments."""
    p = _small(noise=True, ne=3)
    gs, _ = O.ground_state(p, max_steps=50)
    e = O.OracleEnsemble(p)
    e.init(gs)
    e.start_evolution()
    e.evolve(20)
    m, d = e.moments(), e.d
    for alpha in (0.0, 0.5, 2.0, 4.5):
        na, nb = e.ref_rotated_sums(alpha)
        r1, r2 = OBS.rotated(m, d, p.ne, alpha)
        assert na / p.ne == pytest.approx(r1, rel=1e-10, abs=1e-8 * abs(na))
        assert nb / p.ne == pytest.approx(r2, rel=1e-10, abs=1e-8 * abs(nb))
    assert e.ref_visibility() == pytest.approx(OBS.visibility_scan(m, d, p.ne), rel=1e-10)
    np.testing.assert_allclose(e.ref_axial_ratio(), OBS.axial_ratio(e.axial(), d, p.ne), rtol=1e-9, atol=1e-12)
    # analytic visibility bounds the scan (the scan samples 13 angles)
    assert OBS.visibility_scan(m, d, p.ne) <= OBS.visibility(m, d, p.ne) + 1e-12


def test_initial_vacuum_noise_statistics():
    """<|eta|^2> = 1/2 per cell and mode (wigner.cu:211, report.tex:712-723): the Wigner
    population of the pure-noise component averages to zero."""
    p = _small(noise=True, ne=16, losses=False)
    gs, _ = O.ground_state(p, max_steps=20)
    e = O.OracleEnsemble(p)
    e.init(gs)
    tm = e.traj_moments()
    d = e.d
    nb_w = tm[:, 2] - d.cells * d.V / 2
    # each trajectory: sum of cells*... chi-square with 2*cells dof scaled by 1/4 per part
    sd = np.sqrt(d.cells * 2 * 0.25 ** 2 * 2)
    assert abs(nb_w.mean()) < 4 * sd / np.sqrt(p.ne)


def test_injected_noise_equals_philox_noise():
    p = _small(noise=True, ne=2)
    gs, _ = O.ground_state(p, max_steps=20)
    d = O.derive(p)
    noise = np.zeros((p.ne, 2, d.cells), dtype=np.complex128)
    for t in range(p.ne):
        for c in range(d.cells):
            r = O.normals4(p.seed, t, 0, c, 0)
            noise[t, 0, c] = 0.5 * (r[0] + 1j * r[1])
            noise[t, 1, c] = 0.5 * (r[2] + 1j * r[3])
    e1, e2 = O.OracleEnsemble(p), O.OracleEnsemble(p)
    e1.init(gs)
    e2.init(gs, noise)
    for t in range(p.ne):
        np.testing.assert_array_equal(e1.get_state(t), e2.get_state(t))


def test_loss_noise_diffusion_matches_definition():
    """The loss-noise increment has <|d psi|^2> = D dt / dV with
    D11 = (3/2) l111 |a|^4 + (1/2) l12 |b|^2, D22 = (1/2) l12 |a|^2 + l22 |b|^2
    (the diffusion of report.tex:700-720 / poster.tex:276-278 with the rates
    fixed by the deterministic loss drift of wigner_kernel.cu:208-215).
    Checked on the ensemble mean of N_a, N_b after one step against the
    noise-free step, which differs only by the noise."""
    M = 4000
    base = rb87_params(N=20000, grid=(8, 1, 16), ne=M, noise=False, loss_noise=True)
    base.gamma111 *= 1e7
    base.gamma12 *= 1e5
    base.gamma22 *= 1e5
    gs, _ = O.ground_state(copy_params(base, ne=1), max_steps=20)
    quiet = copy_params(base, ne=1, loss_noise=0)
    e0 = O.OracleEnsemble(quiet)
    e0.init(gs); e0.pulse(np.pi / 2)
    e = O.OracleEnsemble(base)
    e.init(gs); e.pulse(np.pi / 2)
    d = e.d
    # the state the nonlinear step sees: x-space after the first half kick
    ab = e0.get_state(0)
    k2 = O.k2_table(d)
    def half(x):
        xk = np.fft.ifftn(x.reshape(d.nvz, d.nvy, d.nvx)).reshape(-1) * np.exp(1j * k2 * d.dt_evo / 2)
        return np.fft.fftn(xk.reshape(d.nvz, d.nvy, d.nvx)).reshape(-1)
    a0, b0 = half(ab[0]), half(ab[1])
    na0, nb0 = np.abs(a0) ** 2, np.abs(b0) ** 2
    dNa = d.dt_evo * (1.5 * d.l111 * (na0 ** 2).sum() + 0.5 * d.l12 * nb0.sum())
    dNb = d.dt_evo * (0.5 * d.l12 * na0.sum() + d.l22 * nb0.sum())
    e0.evolve(1); e.evolve(1)
    q = e0.moments()
    tm = e.traj_moments()
    ex_a, ex_b = tm[:, 1].mean() - q[1], tm[:, 2].mean() - q[2]
    se_a, se_b = tm[:, 1].std() / np.sqrt(M), tm[:, 2].std() / np.sqrt(M)
    assert abs(ex_a - dNa) < 4 * se_a + 1e-3 * dNa
    assert abs(ex_b - dNb) < 4 * se_b + 1e-3 * dNb
    assert dNa > 10 * se_a and dNb > 10 * se_b      # the test resolves the effect
