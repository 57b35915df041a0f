"""Observables as closed-form functions of the FP64 moments.

For one ensemble the device produces na = sum |a|^2 dV, nb = sum |b|^2 dV and
s = sum conj(a) b dV over its trajectories. A pi/2 rotation about the axis at
angle alpha (halfPiRotate, programs/bec_wigner_3d.cuda/wigner_kernel.cu:344-360)
maps |a|^2 -> (na + nb)/2 + Im(e^{i alpha} conj(a) b), |b|^2 -> (na + nb)/2 -
Im(...), so every observable of the reference follows from (na, nb, s) with
the Wigner term V/(2 dV) per cell (wigner_kernel.cu:283-286) subtracted.
"""
import numpy as np


def wigner_sub(d, ne):
    """sum over cells and trajectories of V/(2 dV) * dV."""
    return ne * d.cells * d.V / 2.0


def populations(m, d, ne):
    """(N1, N2) per trajectory, no pulse."""
    sub = wigner_sub(d, ne)
    return (m[1] - sub) / ne, (m[2] - sub) / ne


def rotated(m, d, ne, alpha):
    """(N1(alpha), N2(alpha)) per trajectory after a final pi/2 about axis alpha."""
    sub = wigner_sub(d, ne)
    im = np.sin(alpha) * m[3] + np.cos(alpha) * m[4]
    return ((m[1] + m[2]) / 2 + im - sub) / ne, ((m[1] + m[2]) / 2 - im - sub) / ne


def visibility(m, d, ne):
    """2 |<psi1|psi2>| / (N1 + N2) (report.tex:855-860)."""
    n1, n2 = populations(m, d, ne)
    return 2.0 * np.hypot(m[3], m[4]) / ne / (n1 + n2)


def visibility_scan(m, d, ne):
    """getVisibility (wigner.cu:267-277): max over alpha = 0, 0.5, ... < 2 pi."""
    sub = wigner_sub(d, ne)
    best, alpha = 0.0, 0.0
    while alpha < 2 * np.pi:
        im = np.sin(alpha) * m[3] + np.cos(alpha) * m[4]
        n1 = abs((m[1] + m[2]) / 2 + im - sub)
        n2 = abs((m[1] + m[2]) / 2 - im - sub)
        best = max(best, abs((n1 - n2) / (n1 + n2)))
        alpha += 0.5
    return best


def phase(m):
    """arg <psi1|psi2> in the reference's sign convention."""
    return float(np.arctan2(m[4], m[3]))


def axial_ratio(ax, d, ne):
    """printComponentRatioAxialProjection (wigner.cu:279-303): (a - b)/(a + b) per z after halfPiRotate(0).
    ax[z] = (na(z), nb(z), Re s(z), Im s(z))."""
    sub = ne * d.nvx * d.nvy * d.V / 2.0
    pa = (ax[:, 0] + ax[:, 1]) / 2 + ax[:, 3] - sub
    pb = (ax[:, 0] + ax[:, 1]) / 2 - ax[:, 3] - sub
    return (pa - pb) / (pa + pb)
