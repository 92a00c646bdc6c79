"""HEALPix orientation grids and RELION Euler matrices.

The coarse pass scores every particle against orientations = (HEALPix
direction) x (in-plane psi).  RELION samples directions on a HEALPix grid of a
given order (Nside = 2**order, 12*Nside**2 pixels, RING numbering) and psi at
360/n_psi degree steps.

`pix2ang_ring` is the published RING-scheme pixel-centre formula of
Gorski et al., ApJ 622 (2005) 759, section 4 (north cap, equatorial belt,
south cap).  `euler_matrix` is RELION's ZYZ convention (rot, tilt, psi) as
documented for `Euler_angles2matrix` in RELION's euler.cpp.  The orientation
buffer handed to the kernels holds 9 floats per orientation, row-major, and
the kernels read entries 0,1,3,4,6,7 (reference: src/acc_projectorkernel_impl.h:178-194):
the 3D sample point of image pixel (x, y) is  R @ (x, y, 0).
"""
from __future__ import annotations

import math

import numpy as np


def pix2ang_ring(nside: int) -> tuple[np.ndarray, np.ndarray]:
    """Return (theta, phi) in radians for all 12*nside**2 RING pixel centres."""
    npix = 12 * nside * nside
    ncap = 2 * nside * (nside - 1)
    theta = np.empty(npix)
    phi = np.empty(npix)
    for ipix in range(npix):
        if ipix < ncap:  # north polar cap
            iring = int((1 + math.isqrt(1 + 2 * ipix)) // 2)
            iphi = ipix - 2 * iring * (iring - 1) + 1
            z = 1.0 - iring * iring / (3.0 * nside * nside)
            ph = (iphi - 0.5) * math.pi / (2.0 * iring)
        elif ipix < npix - ncap:  # equatorial belt
            ip = ipix - ncap
            iring = ip // (4 * nside) + nside
            iphi = ip % (4 * nside) + 1
            fodd = 1.0 if ((iring + nside) & 1) else 0.5
            z = (2 * nside - iring) * 2.0 / (3.0 * nside)
            ph = (iphi - fodd) * math.pi / (2.0 * nside)
        else:  # south polar cap
            ip = npix - ipix
            iring = int((1 + math.isqrt(2 * ip - 1)) // 2)
            iphi = 4 * iring + 1 - (ip - 2 * iring * (iring - 1))
            z = -1.0 + iring * iring / (3.0 * nside * nside)
            ph = (iphi - 0.5) * math.pi / (2.0 * iring)
        theta[ipix] = math.acos(max(-1.0, min(1.0, z)))
        phi[ipix] = ph
    return theta, phi


def euler_matrix(rot: np.ndarray, tilt: np.ndarray, psi: np.ndarray) -> np.ndarray:
    """RELION Euler_angles2matrix (angles in radians), shape (..., 3, 3)."""
    ca, sa = np.cos(rot), np.sin(rot)
    cb, sb = np.cos(tilt), np.sin(tilt)
    cg, sg = np.cos(psi), np.sin(psi)
    cc, cs, sc, ss = cb * ca, cb * sa, sb * ca, sb * sa
    a = np.empty(np.broadcast(rot, tilt, psi).shape + (3, 3))
    a[..., 0, 0] = cg * cc - sg * sa
    a[..., 0, 1] = cg * cs + sg * ca
    a[..., 0, 2] = -cg * sb
    a[..., 1, 0] = -sg * cc - cg * sa
    a[..., 1, 1] = -sg * cs + cg * ca
    a[..., 1, 2] = sg * sb
    a[..., 2, 0] = sc
    a[..., 2, 1] = ss
    a[..., 2, 2] = cb
    return a


def orientation_grid(order: int, n_psi: int) -> tuple[np.ndarray, np.ndarray]:
    """Coarse orientation grid: HEALPix(order) directions x n_psi in-plane angles.

    Returns (eulers [O, 9] float32, direction index [O] int) with orientation
    o = dir * n_psi + ipsi.  Each 3x3 block is R = A^T so that R @ (x, y, 0)
    is the 3D Fourier position of image pixel (x, y).
    """
    nside = 2 ** order
    theta, phi = pix2ang_ring(nside)
    psi = np.arange(n_psi) * (2.0 * math.pi / n_psi)
    rot = np.repeat(phi, n_psi)
    tilt = np.repeat(theta, n_psi)
    ps = np.tile(psi, theta.size)
    a = euler_matrix(rot, tilt, ps)
    r = np.swapaxes(a, -1, -2)
    eul = r.reshape(-1, 9).astype(np.float32)
    return eul, np.repeat(np.arange(theta.size), n_psi)


def direction_vectors(order: int) -> np.ndarray:
    """Unit vectors of the HEALPix(order) pixel centres, shape [npix, 3]."""
    theta, phi = pix2ang_ring(2 ** order)
    st = np.sin(theta)
    return np.stack([st * np.cos(phi), st * np.sin(phi), np.cos(theta)], axis=1)
