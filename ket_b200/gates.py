"""Gate matrices: the formulas of the reference's src/gates.ts:11-208.

Each function returns a nested tuple of Python complex numbers in the
reference's row-major layout (2x2, or 4x4 with the first qubit as MSB).
Entries are built from the same expressions (same operand order, same
1/sqrt(2) constant) so they match the reference to the last bit wherever the
platform's cos/sin do.
"""
from __future__ import annotations

import math

sq2 = 1 / math.sqrt(2)  # gates.ts:11

ZERO = complex(0, 0)
ONE = complex(1, 0)


def c(re: float, im: float = 0.0) -> complex:
    return complex(re, im)


Id = ((ONE, ZERO), (ZERO, ONE))
H = ((c(sq2), c(sq2)), (c(sq2), c(-sq2)))
X = ((ZERO, ONE), (ONE, ZERO))
Y = ((ZERO, c(0, -1)), (c(0, 1), ZERO))
Z = ((ONE, ZERO), (ZERO, c(-1)))
S = ((ONE, ZERO), (ZERO, c(0, 1)))
Si = ((ONE, ZERO), (ZERO, c(0, -1)))
T = ((ONE, ZERO), (ZERO, c(sq2, sq2)))
Ti = ((ONE, ZERO), (ZERO, c(sq2, -sq2)))
V = ((c(.5, .5), c(.5, -.5)), (c(.5, -.5), c(.5, .5)))
Vi = ((c(.5, -.5), c(.5, .5)), (c(.5, .5), c(.5, -.5)))


def Rx(theta: float):  # gates.ts:25-29
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(co), c(0, -si)), (c(0, -si), c(co)))


def Ry(theta: float):  # gates.ts:32-36
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(co, 0), c(-si)), (c(si), c(co)))


def Rz(theta: float):  # gates.ts:39-43
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(co, -si), ZERO), (ZERO, c(co, si)))


R2 = Rz(math.pi / 2)
R4 = Rz(math.pi / 4)
R8 = Rz(math.pi / 8)


def U3(theta: float, phi: float, lam: float):  # gates.ts:71-77
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(co), c(-si * math.cos(lam), -si * math.sin(lam))),
            (c(si * math.cos(phi), si * math.sin(phi)), c(co * math.cos(phi + lam), co * math.sin(phi + lam))))


def U2(phi: float, lam: float):
    return U3(math.pi / 2, phi, lam)


def U1(lam: float):  # gates.ts:89-90
    return ((ONE, ZERO), (ZERO, c(math.cos(lam), math.sin(lam))))


def Xx(theta: float):  # gates.ts:99-107
    co, ni = c(math.cos(theta / 2)), c(0, -math.sin(theta / 2))
    return ((co, ZERO, ZERO, ni), (ZERO, co, ni, ZERO), (ZERO, ni, co, ZERO), (ni, ZERO, ZERO, co))


def Yy(theta: float):  # gates.ts:112-122
    co, ni, pi = c(math.cos(theta / 2)), c(0, -math.sin(theta / 2)), c(0, math.sin(theta / 2))
    return ((co, ZERO, ZERO, pi), (ZERO, co, ni, ZERO), (ZERO, ni, co, ZERO), (pi, ZERO, ZERO, co))


def Zz(theta: float):  # gates.ts:129-138
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    m, p = c(co, -si), c(co, si)
    return ((m, ZERO, ZERO, ZERO), (ZERO, p, ZERO, ZERO), (ZERO, ZERO, p, ZERO), (ZERO, ZERO, ZERO, m))


def Xy(theta: float):  # gates.ts:145-153
    co, is_ = c(math.cos(theta / 2)), c(0, math.sin(theta / 2))
    return ((ONE, ZERO, ZERO, ZERO), (ZERO, co, is_, ZERO), (ZERO, is_, co, ZERO), (ZERO, ZERO, ZERO, ONE))


ISwap = Xy(math.pi)
SrSwap = Xy(math.pi / 2)


def Gpi(phi: float):  # gates.ts:166-169
    co, si = math.cos(phi), math.sin(phi)
    return ((ZERO, c(co, -si)), (c(co, si), ZERO))


def Gpi2(phi: float):  # gates.ts:179-184
    co, si = math.cos(phi), math.sin(phi)
    return ((c(sq2), c(-sq2 * si, -sq2 * co)), (c(sq2 * si, -sq2 * co), c(sq2)))


def Ms(phi0: float, phi1: float):  # gates.ts:194-208
    sp, cp = math.sin(phi0 + phi1), math.cos(phi0 + phi1)
    sd, cd = math.sin(phi0 - phi1), math.cos(phi0 - phi1)
    return ((c(sq2), ZERO, ZERO, c(-sp * sq2, -cp * sq2)),
            (ZERO, c(sq2), c(-sd * sq2, -cd * sq2), ZERO),
            (ZERO, c(sd * sq2, -cd * sq2), c(sq2), ZERO),
            (c(sp * sq2, -cp * sq2), ZERO, ZERO, c(sq2)))


# Derivatives d/dtheta of the one-parameter gate families, used by the adjoint
# gradient.  Each is the entry-wise derivative of the formula above.
def dRx(theta):
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(-si / 2), c(0, -co / 2)), (c(0, -co / 2), c(-si / 2)))


def dRy(theta):
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(-si / 2), c(-co / 2)), (c(co / 2), c(-si / 2)))


def dRz(theta):
    co, si = math.cos(theta / 2), math.sin(theta / 2)
    return ((c(-si / 2, -co / 2), ZERO), (ZERO, c(-si / 2, co / 2)))


def dU1(lam):
    return ((ZERO, ZERO), (ZERO, c(-math.sin(lam), math.cos(lam))))
