"""Plain numpy restatement of the reference's fast-multipole conventions (test infrastructure,
the checker of the fixtures and of the device multipole kernels; never part of the product).

  regular(p, x)        R_n^m(x) = r^n P~_n^|m|(cos t) e^{i m phi}, P~_n^m = (-1)^m
                       sqrt((n-m)!/(n+m)!) P_n^m, R_n^-m = conj(R_n^m), index n(n+1)+m
                       (KFMMath.cc:219-330 ALP_nm, 1056-1123 RegularSolidHarmonic_Cart_Array)
  moments(verts, o, p) moments of unit total charge spread uniformly over a wire / triangle /
                       rectangle: the average over the element of conj(R_n^m(y - o))
                       (KFMElectrostaticMultipoleCalculatorAnalytic.cc:169-224 normalises the
                       analytic integral by the area or length), by a Gauss-Legendre cubature that
                       is exact for these polynomials
  local_field(...)     phi = sum_n [L_n0 R_n0 + 2 sum_m>0 Re(L_nm R_nm)] / (4 pi eps0) and its
                       gradient by central differences
                       (KFMElectrostaticLocalCoefficientFieldCalculator.cc:285-310)
  response(kind, ...)  the M2M / M2L / L2L response functions (KFMResponseKernel_3DLaplaceM2M.cc,
                       ...M2L.cc, ...L2L.cc), del = source - target origin
"""

from __future__ import annotations

from math import factorial, sqrt

import numpy as np
from scipy.special import lpmv


def _alp(n, m, x):
    return sqrt(factorial(n - m) / factorial(n + m)) * lpmv(m, n, x)


def regular(p: int, x) -> np.ndarray:
    x = np.asarray(x, np.float64)
    r = float(np.linalg.norm(x))
    ct = x[2] / r if r > 0 else 0.0
    ph = float(np.arctan2(x[1], x[0]))
    out = np.zeros((p + 1) ** 2, complex)
    for n in range(p + 1):
        for m in range(n + 1):
            v = r ** n * _alp(n, m, ct) * np.exp(1j * m * ph)
            out[n * (n + 1) + m] = v
            out[n * (n + 1) - m] = np.conj(v)
    return out


def irregular(p: int, x) -> np.ndarray:
    r = float(np.linalg.norm(x))
    R = regular(p, x)
    for n in range(p + 1):
        R[n * n:(n + 1) ** 2] /= r ** (2 * n + 1)
    return R


def moments(verts, origin, p: int) -> np.ndarray:
    v = np.asarray(verts, np.float64)
    o = np.asarray(origin, np.float64)
    q = p // 2 + 2
    x, w = np.polynomial.legendre.leggauss(q)
    u, wu = (x + 1) / 2, w / 2
    M = np.zeros((p + 1) ** 2, complex)
    if len(v) == 2:
        for a, wa in zip(u, wu):
            M += wa * np.conj(regular(p, v[0] + a * (v[1] - v[0]) - o))
    elif len(v) == 3:
        for a, wa in zip(u, wu):
            for b, wb in zip(u, wu):
                y = v[0] + a * (v[1] - v[0]) + b * (1 - a) * (v[2] - v[0])
                M += 2 * wa * wb * (1 - a) * np.conj(regular(p, y - o))
    else:
        for a, wa in zip(u, wu):
            for b, wb in zip(u, wu):
                y = v[0] + a * (v[1] - v[0]) + b * (v[3] - v[0])
                M += wa * wb * np.conj(regular(p, y - o))
    return M


def local_field(p: int, origin, coeff, P, one_over_four_pi_eps0: float, h: float = 1e-6) -> np.ndarray:
    """coeff: m >= 0 coefficients in the index l(l+1)/2 + m; returns n x (Ex, Ey, Ez, phi)."""
    o = np.asarray(origin, np.float64)

    def phi(x):
        R = regular(p, x - o)
        s = 0.0
        for n in range(p + 1):
            for m in range(n + 1):
                term = (coeff[n * (n + 1) // 2 + m] * R[n * (n + 1) + m]).real
                s += term if m == 0 else 2 * term
        return one_over_four_pi_eps0 * s

    out = []
    for x in np.asarray(P, np.float64).reshape(-1, 3):
        g = [(phi(x + h * e) - phi(x - h * e)) / (2 * h) for e in np.eye(3)]
        out.append([-g[0], -g[1], -g[2], phi(x)])
    return np.array(out)


def _a(m, n):
    return (-1) ** n / sqrt(factorial(n - m) * factorial(n + m))


def response(kind: int, p: int, source_origin, target_origin) -> np.ndarray:
    d = np.asarray(source_origin, np.float64) - np.asarray(target_origin, np.float64)
    S = (p + 1) ** 2
    C = np.zeros((S, S), complex)
    H = irregular(2 * p, d) if kind == 1 else regular(p, d)
    for j in range(p + 1):
        for k in range(-j, j + 1):
            for n in range(p + 1):
                for m in range(-n, n + 1):
                    if kind == 0:
                        npr, mpr = j - n, k - m
                        if npr < 0 or abs(mpr) > npr:
                            continue
                        pre = 1.0
                        if (k - mpr) * mpr < 0:
                            pre *= (-1) ** min(abs(k - mpr), abs(mpr))
                        pre *= _a(mpr, npr) * _a(k - mpr, j - npr) / _a(k, j)
                        v = pre * H[npr * (npr + 1) - mpr]
                    elif kind == 1:
                        f = (-1) ** n
                        if k * m > 0 and min(abs(m), abs(k)) % 2 == 1:
                            f = -f
                        f *= _a(m, n) * _a(k, j) / _a(m - k, j + n)
                        v = f * H[(j + n) * (j + n + 1) + (m - k)]
                    else:
                        if n < j or abs(m - k) > n - j:
                            continue
                        pref = (-1) ** (n + j) * (1j) ** (abs(m) - abs(m - k) - abs(k))
                        pref *= _a(m - k, n - j) * _a(k, j) / _a(m, n)
                        v = pref * H[(n - j) * (n - j + 1) + (m - k)]
                    C[j * (j + 1) + k, n * (n + 1) + m] = v
    return C
