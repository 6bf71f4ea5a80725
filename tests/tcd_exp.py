"""The reference's recorded time-dependent known answer (TCD2D, example exp.h).

ReadIn/tcd2d.out:485-543 is a run of 2DPrograms/TCD2D_ParMooN.C on the unit square with
32 x 32 Q1 cells (1089 DOFs, 961 active), Gauss3, Galerkin, Crank-Nicolson (TIME_DISC 2,
theta1..theta4 = 0.5), tau = 0.05, PE_NR 1, and the example Examples/TCD_2D/exp.h:
u = exp(t) sin(2 pi x) sin(2 pi y) (lines 31-41), eps = 1, b = (1, -1), c = 1 and the matching
right-hand side (lines 66-91), Dirichlet 0.  The run prints the L2 and H1-semi errors of the
initial interpolant and of every step; they are reproduced here to all printed digits.
"""
import numpy as np

TAU = 0.05
THETA = (0.5, 0.5, 0.5, 0.5)
# (time, L2, H1-semi) as printed, ReadIn/tcd2d.out:490-543
KNOWN = [
    (0.00, "3.360188e-03", "2.521492e-01"),
    (0.05, "1.541462e-03", "2.647214e-01"),
    (0.10, "2.207736e-03", "2.782276e-01"),
    (0.15, "2.116156e-03", "2.924973e-01"),
    (0.20, "2.287663e-03", "3.074884e-01"),
    (0.25, "2.385831e-03", "3.232560e-01"),
    (0.30, "2.513170e-03", "3.398282e-01"),
    (0.35, "2.641077e-03", "3.572524e-01"),
    (0.40, "2.776346e-03", "3.755686e-01"),
    (0.45, "2.919008e-03", "3.948248e-01"),
    (0.50, "3.068387e-03", "4.150676e-01"),
]


def coeff_table(xq, t):
    """eps, b1, b2, b3, c, f of exp.h at quadrature points xq (..., 2), time t."""
    x, y = xq[..., 0], xq[..., 1]
    eps, b1, b2, c = 1.0, 1.0, -1.0, 1.0
    e = np.exp(t)
    s = np.sin(2 * np.pi * x) * np.sin(2 * np.pi * y)
    sx = np.cos(2 * np.pi * x) * np.sin(2 * np.pi * y)
    sy = np.sin(2 * np.pi * x) * np.cos(2 * np.pi * y)
    f = e * s - eps * e * 4 * np.pi ** 2 * (-s - s) + b1 * e * 2 * np.pi * sx + b2 * e * 2 * np.pi * sy + c * e * s
    tab = np.zeros(xq.shape[:-1] + (6,))
    tab[..., 0], tab[..., 1], tab[..., 2], tab[..., 4], tab[..., 5] = eps, b1, b2, c, f
    return tab


def initial(xyz):
    """the interpolant of the initial condition (exp.h:55-62) at the DOF coordinates"""
    return np.sin(2 * np.pi * xyz[:, 0]) * np.sin(2 * np.pi * xyz[:, 1])


def fmt(e):
    return f"{e[0]:.6e}", f"{e[1]:.6e}"
