"""Cell quadrature and initial states on the host (setup only, vectorised numpy).

Cell integrals use the reconstruction's cell schemes: Hammer TRI_4 and Gauss
QUAD_9 (DNDS_FV_VR.cpp:37,42; tables DNDS_Elements.hpp:326-430).
"""
from __future__ import annotations

import numpy as np

from .mesh import Mesh

_A = np.sqrt(0.6)
_L3 = (np.array([-_A, 0.0, _A]), np.array([5.0, 8.0, 5.0]) / 9.0)
_TRI4 = (
    np.array([[1.0 / 3.0, 1.0 / 3.0], [0.6, 0.2], [0.2, 0.6], [0.2, 0.2]]),
    np.array([-27.0, 25.0, 25.0, 25.0]) / 96.0,
)
_Q9P = np.array([[_L3[0][i], _L3[0][j]] for j in range(3) for i in range(3)])
_Q9W = np.array([_L3[1][i] * _L3[1][j] for j in range(3) for i in range(3)])


def cell_quadrature(mesh: Mesh):
    """Physical gauss points [N, 9, 2] and weights w*detJ [N, 9] (zero-padded for triangles)."""
    n = mesh.n_cells
    pts = np.zeros((n, 9, 2))
    wts = np.zeros((n, 9))
    cn = mesh.cell_nodes
    xy = mesh.node_xy
    tri = cn[:, 3] < 0
    it = np.nonzero(tri)[0]
    if it.size:
        p0, p1, p2 = xy[cn[it, 0]], xy[cn[it, 1]], xy[cn[it, 2]]
        det = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p1[:, 1] - p0[:, 1]) * (p2[:, 0] - p0[:, 0])
        for g, (xi, eta) in enumerate(_TRI4[0]):
            pts[it, g] = p0 * (1 - xi - eta) + p1 * xi + p2 * eta
            wts[it, g] = det * _TRI4[1][g]
    iq = np.nonzero(~tri)[0]
    if iq.size:
        P = [xy[cn[iq, k]] for k in range(4)]
        for g, (xi, eta) in enumerate(_Q9P):
            N = np.array([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta), (1 - xi) * (1 + eta)]) * 0.25
            dxi = np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)]) * 0.25
            deta = np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)]) * 0.25
            x = sum(N[k] * P[k] for k in range(4))
            jx = sum(dxi[k] * P[k] for k in range(4))
            jy = sum(deta[k] * P[k] for k in range(4))
            pts[iq, g] = x
            wts[iq, g] = (jx[:, 0] * jy[:, 1] - jx[:, 1] * jy[:, 0]) * _Q9W[g]
    return pts, wts


def cell_average(mesh: Mesh, fn) -> np.ndarray:
    """Cell averages of fn(x, y) -> [..., nv] using the cell quadrature."""
    pts, wts = cell_quadrature(mesh)
    vals = fn(pts[..., 0], pts[..., 1])  # [N, 9, nv]
    vol = wts.sum(1)
    return np.einsum("ng,ngv->nv", wts, vals) / vol[:, None]


def isentropic_vortex_state(x, y, t=0.0, gamma=1.4, taper=True, period=10.0):
    """Conservative isentropic-vortex state (DNDS_FV_EulerSolver.hpp:536-582),
    centre (5,5) moving with (1,1); chi = 5; rm = 8 taper. Periodic images are folded."""
    chi, rm = 5.0, 8.0
    xc = np.fmod(5.0 + t, period)
    yc = np.fmod(5.0 + t, period)
    dx = x - xc
    dy = y - yc
    if t != 0.0:
        dx = dx - period * np.round(dx / period)
        dy = dy - period * np.round(dy / period)
    r2 = dx * dx + dy * dy
    tp = (1.0 - 1.0 / np.exp(np.maximum(rm * rm - r2, 0.0))) if taper else 1.0
    dT = -(gamma - 1.0) / (8.0 * gamma * np.pi ** 2) * chi ** 2 * np.exp(1.0 - r2) * tp
    dux = chi / 2.0 / np.pi * np.exp((1.0 - r2) / 2.0) * -dy * tp
    duy = chi / 2.0 / np.pi * np.exp((1.0 - r2) / 2.0) * dx * tp
    T = dT + 1.0
    ux = dux + 1.0
    uy = duy + 1.0
    rho = T ** (1.0 / (gamma - 1.0))
    p = T * rho
    E = 0.5 * (ux * ux + uy * uy) * rho + p / (gamma - 1.0)
    return np.stack([rho, rho * ux, rho * uy, E], axis=-1)


def isentropic_vortex(mesh: Mesh, t=0.0, gamma=1.4) -> np.ndarray:
    return cell_average(mesh, lambda x, y: isentropic_vortex_state(x, y, t, gamma))


def quadrant_states(mesh: Mesh, states, xs=0.8, ys=0.8, gamma=1.4) -> np.ndarray:
    """Piecewise-constant four-quadrant state by cell barycentre; states = NE, NW, SW, SE (rho,u,v,p)."""
    pts, wts = cell_quadrature(mesh)
    vol = wts.sum(1)
    bx = (pts[..., 0] * wts).sum(1) / vol
    by = (pts[..., 1] * wts).sum(1) / vol
    k = np.where(bx > xs, np.where(by > ys, 0, 3), np.where(by > ys, 1, 2))
    q = np.array(states, dtype=np.float64)
    rho, u, v, p = q[k, 0], q[k, 1], q[k, 2], q[k, 3]
    return np.stack([rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)], axis=1)
