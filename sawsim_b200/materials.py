"""Material tensors for the sweep backend (host setup, O(1) per material).

Stress-charge form, Voigt order ``xx, yy, zz, yz, xz, xy``: stiffness ``C``
(6x6, Pa), piezoelectric ``e`` (3x6, C/m^2), permittivity ``eps`` (3x3, F/m),
density ``rho`` (kg/m^3).

Follows the reference's crystal-class builders (``src/sawsim/crystal.py:30-78``)
and its intrinsic ZXZ Euler rotation with the Bond-matrix transform
(``src/sawsim/saw2d/materials.py:28-71``, ``:250-265``), including the order in
which the angle conversion is evaluated (degrees * pi / 180, not deg2rad),
because the Hex27 regression is sensitive to 1-ulp changes there.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

EPS0 = 8.8541878128e-12          # crystal builder value (src/sawsim/crystal.py:10)
EPS0_LEGACY = 8.854e-12          # legacy value (src/sawsim/saw2d/materials.py:15)


@dataclass
class Material:
    """One material in device axes (already rotated)."""

    rho: float
    C: np.ndarray
    e: np.ndarray
    eps: np.ndarray


def isotropic(E: float, nu: float, rho: float, eps_r: float = 1.0) -> Material:
    """Isotropic solid from Young's modulus (Pa) and Poisson ratio (crystal.py:39-47)."""
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    for i in range(3):
        C[i, i] = lam + 2 * mu
        C[i + 3, i + 3] = mu
    return Material(float(rho), C, np.zeros((3, 6)), np.eye(3) * eps_r * EPS0)


def cubic(c11: float, c12: float, c44: float, rho: float, eps_r: float = 1.0) -> Material:
    """Cubic m3m crystal, constants in Pa (crystal.py:48-54)."""
    C = np.zeros((6, 6))
    C[:3, :3] = c12
    for i in range(3):
        C[i, i] = c11
        C[i + 3, i + 3] = c44
    return Material(float(rho), C, np.zeros((3, 6)), np.eye(3) * eps_r * EPS0)


def trigonal_3m(k: dict, rho: float) -> Material:
    """3m crystal (LiNbO3/LiTaO3 class) in crystal axes; C in Pa, e in C/m^2, eps relative.

    Keys: C11 C12 C13 C14 C33 C44 e15 e22 e31 e33 eps11 eps33. C66 = (C11-C12)/2,
    +C14 / +e22 sign convention of crystal.py:55-77.
    """
    c11, c12, c13, c33, c44 = (float(k[x]) for x in ('C11', 'C12', 'C13', 'C33', 'C44'))
    c14 = float(k['C14'])
    C = np.zeros((6, 6))
    C[0, 0] = C[1, 1] = c11
    C[0, 1] = C[1, 0] = c12
    C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = c13
    C[2, 2] = c33
    C[3, 3] = C[4, 4] = c44
    C[5, 5] = (c11 - c12) / 2
    C[0, 3] = C[3, 0] = c14
    C[1, 3] = C[3, 1] = -c14
    C[4, 5] = C[5, 4] = c14
    e = np.zeros((3, 6))
    e[0, 4] = e[1, 3] = k['e15']
    e[2, 0] = e[2, 1] = k['e31']
    e[2, 2] = k['e33']
    e[0, 5] = -k['e22']
    e[1, 0] = -k['e22']
    e[1, 1] = k['e22']
    eps = np.zeros((3, 3))
    eps[0, 0] = eps[1, 1] = k['eps11'] * EPS0
    eps[2, 2] = k['eps33'] * EPS0
    return Material(float(rho), C, e, eps)


def rotation_matrix(angles_deg) -> np.ndarray:
    """Intrinsic ZXZ rotation A = Rz(alpha) Rx(beta) Rz(gamma), angles in degrees.

    Same evaluation order as src/sawsim/saw2d/materials.py:259-265.
    """
    alpha, beta, gamma = np.asarray(angles_deg, dtype=float) * np.pi / 180.0

    def rz(t):
        c, s = np.cos(t), np.sin(t)
        return np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])

    c, s = np.cos(beta), np.sin(beta)
    rx = np.array([[1, 0, 0], [0, c, -s], [0, s, c]])
    return rz(alpha) @ rx @ rz(gamma)


def bond_matrix(a: np.ndarray) -> np.ndarray:
    """6x6 Bond stress transformation for a 3x3 rotation ``a`` (materials.py:48-66)."""
    M = np.empty((6, 6), dtype=a.dtype)
    M[:3, :3] = a ** 2
    M[:3, 3] = 2 * a[:, 1] * a[:, 2]
    M[:3, 4] = 2 * a[:, 0] * a[:, 2]
    M[:3, 5] = 2 * a[:, 0] * a[:, 1]
    M[3, :3] = a[1, :] * a[2, :]
    M[4, :3] = a[0, :] * a[2, :]
    M[5, :3] = a[0, :] * a[1, :]
    M[3, 3] = a[1, 1] * a[2, 2] + a[1, 2] * a[2, 1]
    M[3, 4] = a[1, 0] * a[2, 2] + a[1, 2] * a[2, 0]
    M[3, 5] = a[1, 1] * a[2, 0] + a[1, 0] * a[2, 1]
    M[4, 3] = a[0, 1] * a[2, 2] + a[0, 2] * a[2, 1]
    M[4, 4] = a[0, 2] * a[2, 0] + a[0, 0] * a[2, 2]
    M[4, 5] = a[0, 0] * a[2, 1] + a[0, 1] * a[2, 0]
    M[5, 3] = a[0, 1] * a[1, 2] + a[0, 2] * a[1, 1]
    M[5, 4] = a[0, 2] * a[1, 0] + a[0, 0] * a[1, 2]
    M[5, 5] = a[0, 0] * a[1, 1] + a[0, 1] * a[1, 0]
    return M


def rotate(mat: Material, angles_deg) -> Material:
    """Rotate crystal-axis tensors into device axes: C'=M C M^T, e'=a e M^T, eps'=a eps a^T."""
    a = rotation_matrix(angles_deg)
    M = bond_matrix(a)
    return Material(mat.rho, M @ mat.C @ M.T, a @ mat.e @ M.T, a @ mat.eps @ a.T)


def project_xy_plane_strain(mat: Material) -> Material:
    """uz = 0, Ez = 0 projection onto the device xy plane (materials.py:281-290)."""
    s = [0, 1, 5]
    el = [0, 1]
    return Material(mat.rho, mat.C[np.ix_(s, s)], mat.e[np.ix_(el, s)], mat.eps[np.ix_(el, el)])


def project_xz_plane_strain(mat: Material) -> Material:
    """The TC-SAW projection (materials.py:303-308): the source frame's xz plane
    becomes the mesh's xy plane (strain rows xx, zz, xz; fields x, z), after the
    source-frame rotation; the result is lifted like an xy projection."""
    s = [0, 2, 4]
    el = [0, 2]
    return Material(mat.rho, mat.C[np.ix_(s, s)], mat.e[np.ix_(el, s)], mat.eps[np.ix_(el, el)])


def lift_plane_strain(mat: Material) -> Material:
    """Zero-filled 6x6/3x6/3x3 tensors from projected 3x3/2x3/2x2 ones (piezo_fem.py:389-401)."""
    if mat.C.shape != (3, 3) or mat.e.shape != (2, 3) or mat.eps.shape != (2, 2):
        raise ValueError('plane-strain lift needs projected xy tensors: C 3x3, e 2x3, eps 2x2')
    s = [0, 1, 5]
    el = [0, 1]
    C = np.zeros((6, 6), dtype=mat.C.dtype)
    e = np.zeros((3, 6), dtype=mat.e.dtype)
    eps = np.zeros((3, 3), dtype=mat.eps.dtype)
    C[np.ix_(s, s)] = mat.C
    e[np.ix_(el, s)] = mat.e
    eps[np.ix_(el, el)] = mat.eps
    return Material(mat.rho, C, e, eps)


def seeded_3m(seed: int = 0, rho: float = 4700.0):
    """Seeded synthetic 3m piezo crystal and ZXZ Euler triple.

    C11, C33, C44, C66 uniform in 0.5-2.5e11 Pa (C12 = C11 - 2 C66), C13 and C14
    drawn so that C is positive definite (reject and redraw); e15, e22, e31, e33
    uniform in 0.1-4 C/m^2 with random signs; eps11, eps33 uniform in 28-45;
    Euler angles uniform in [-180, 180) degrees.

    Returns ``(crystal_axes_material, euler_deg)``.
    """
    rng = np.random.default_rng(seed)
    while True:
        c11, c33, c44, c66 = rng.uniform(0.5e11, 2.5e11, 4)
        c12 = c11 - 2 * c66
        c13 = rng.uniform(-0.6, 0.6) * np.sqrt(c11 * c33)
        c14 = rng.uniform(-0.3, 0.3) * np.sqrt(c11 * c44)
        k = dict(C11=c11, C12=c12, C13=c13, C14=c14, C33=c33, C44=c44)
        m = trigonal_3m(dict(k, e15=0, e22=0, e31=0, e33=0, eps11=1, eps33=1), rho)
        if np.linalg.eigvalsh(m.C).min() > 0.05e11:
            break
    mags = rng.uniform(0.1, 4.0, 4) * rng.choice([-1.0, 1.0], 4)
    k.update(e15=mags[0], e22=mags[1], e31=mags[2], e33=mags[3])
    k.update(eps11=rng.uniform(28, 45), eps33=rng.uniform(28, 45))
    euler = rng.uniform(-180.0, 180.0, 3)
    return trigonal_3m(k, rho), euler


def al() -> Material:
    """Isotropic Al electrode: E 70 GPa, nu 0.35, rho 2700."""
    return isotropic(70e9, 0.35, 2700.0, 1.0)


def sio2() -> Material:
    """Isotropic SiO2: E 72 GPa, nu 0.17, rho 2200, eps_r 3.9."""
    return isotropic(72e9, 0.17, 2200.0, 3.9)


def si_cubic() -> Material:
    """Cubic Si backing: c11 165.7, c12 63.9, c44 79.6 GPa, rho 2330, eps_r 11.7."""
    return cubic(165.7e9, 63.9e9, 79.6e9, 2330.0, 11.7)


def poly_si() -> Material:
    """Isotropic poly-Si: E 169 GPa, nu 0.22, rho 2320, eps_r 4.5."""
    return isotropic(169e9, 0.22, 2320.0, 4.5)


def pack(materials, ndisp: int = 3):
    """Flatten a material list into the C-ABI arrays.

    ``ndisp == 2`` (plane strain) accepts projected tensors and lifts them.
    Returns ``(rho[n], C[n,6,6,2], e[n,3,6,2], eps[n,3,3,2])`` float64 arrays with
    the complex parts interleaved (re, im).
    """
    mats = [lift_plane_strain(m) if ndisp == 2 and m.C.shape == (3, 3) else m for m in materials]
    rho = np.array([m.rho for m in mats], dtype=np.float64)

    def cplx(a):
        a = np.asarray(a, dtype=np.complex128)
        return np.ascontiguousarray(np.stack([a.real, a.imag], axis=-1))

    C = cplx(np.stack([m.C for m in mats]))
    e = cplx(np.stack([m.e for m in mats]))
    eps = cplx(np.stack([m.eps for m in mats]))
    return rho, C, e, eps
