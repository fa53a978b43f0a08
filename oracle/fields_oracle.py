"""Plane-wave excitation restated from the reference (TEST INFRASTRUCTURE ONLY).

``test_fields`` (codes/GPU_implementation/seed/compres_single_block_spheres_for_sweep2.jl:60-85):
incidence direction k_i = -(sin th cos ph, sin th sin ph, cos th), polarisation
e_i = cos(rot) (-sin ph, cos ph, 0) + sin(rot) (cos th cos ph, cos th sin ph, -sin th), and per RWG
E_m = l_m / 2 [ e_i . rho+_c exp(-jk k_i . c(T+)) + e_i . rho-_c exp(-jk k_i . c(T-)) ] with
rho+_c = c(T+) - v+ and rho-_c = v- - c(T-). As in the reference, th = theta pi / 180 and
rot = rot pi / 180 but ph = phi / 180 (no factor pi). Also H_m of the same routine.
"""
from __future__ import annotations

import numpy as np


def test_fields(mesh, theta_i: float, phi_i: float, rot_i: float, k: float, eta: float):
    th = theta_i * np.pi / 180
    ph = phi_i / 180
    rot = rot_i * np.pi / 180
    k_i = -np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
    e_i = (np.cos(rot) * np.array([-np.sin(ph), np.cos(ph), 0.0])
           + np.sin(rot) * np.array([np.cos(th) * np.cos(ph), np.cos(th) * np.sin(ph), -np.sin(th)]))
    h_i = np.cross(k_i, e_i)
    Tp = mesh.edges[0].astype(int) - 1
    Tm = mesh.edges[1].astype(int) - 1
    cp, cm = mesh.cent[:, Tp], mesh.cent[:, Tm]
    pp = np.exp(-1j * k * (k_i @ cp))
    pm = np.exp(-1j * k * (k_i @ cm))
    rp = cp - mesh.vertex[:, mesh.edges[2].astype(int) - 1]
    rm = mesh.vertex[:, mesh.edges[3].astype(int) - 1] - cm
    E = mesh.ln * ((e_i @ rp) * pp + (e_i @ rm) * pm) / 2
    up, um = mesh.un[:, Tp], mesh.un[:, Tm]
    H = mesh.ln * ((h_i @ np.cross(rp.T, up.T).T) * pp + (h_i @ np.cross(rm.T, um.T).T) * pm) / (2 * eta)
    return E, H
