"""Python restatements of the reference's deterministic example projects.

Each builder returns the parameter list that the reference's example function
passes to xsim/xspde, with the MATLAB anonymous functions rewritten as NumPy
callables for the oracle (oracle/xspde_ref.py).  Sources, in the reference:
Examples/SPDE_2D/Soliton.m, Characteristic.m, SolitonAv.m, SolitonDerivS.m, SolitonDerivN.m,
Boundaries2.m, Peregrine.m; Examples/SPDE_3D/GaussianAv2D.m,
GaussianKinetic.m; Examples/SPDE_nD/GaussianAv4D.m, Gaussian3D.m.
"""
import numpy as np

from oracle import xspde_ref as X


def sech(x):
    return 1 / np.cosh(x)


def soliton():
    return [dict(dimensions=2, checks=0, order=2, initial=lambda v, p: sech(p.x),
                 deriv=lambda a, w, p: 1j * a * (np.conj(a) * a),
                 linear=lambda p: 0.5j * (p.Dx ** 2 - 1.0), compare=lambda p: sech(p.x))]


def characteristic():
    return [dict(dimensions=2, initial=lambda w, p: sech(2 * (p.x + 2.5)), linear=lambda p: -p.Dx,
                 points=[51, 35], observe=[lambda a, p: a, lambda a, p: a ** 2], axes=[None, [0, 18]],
                 compare=[None, lambda p: sech(2 * (p.t - 2.5)) ** 2])]


def soliton_av():
    return [dict(dimensions=2,
                 observe=[lambda a, p: X.Ave(np.real(a), p.dx, p), lambda a, p: X.Int(np.real(a), p.dx, p)],
                 initial=lambda v, p: sech(p.x), deriv=lambda a, w, p: 1j * a * (np.conj(a) * a),
                 linear=lambda p: 0.5j * (p.Dx ** 2 - 1.0),
                 compare=[lambda p: np.pi / 10 + 0 * p.t, lambda p: np.pi + 0 * p.t])]


def _g2(p):
    sig = 1 + (p.t / 10) ** 2
    return sig ** -1 * np.exp(-(p.x ** 2 + p.y ** 2) / sig)


def gaussian_av2d():
    I = lambda a, p: a * np.conj(a)
    return [dict(dimensions=3, initial=lambda v, p: np.exp(-0.5 * (p.x ** 2 + p.y ** 2)),
                 deriv=lambda a, w, p: np.zeros(a.shape),
                 observe=[I, lambda a, p: X.Ave(I(a, p), p.dx, p), lambda a, p: X.Int(I(a, p), p.dx, p), I],
                 linear=lambda p: 1j * 0.05 * (p.Dx ** 2 + p.Dy ** 2), transforms=[0, 0, 0, [0, 1, 1]],
                 compare=[_g2, None, None, lambda r: 1], axes=[None, None, None, [0, -1, -1]])]


def gaussian_kinetic():
    y0, x0 = 0.235, 3.3
    A = lambda a: abs(a) ** 2
    return [dict(dimensions=3, fields=1, ranges=[5, 200, 6], points=[49, 70, 34],
                 initial=lambda v, p: np.sqrt(np.exp(-p.x ** 2 / x0 ** 2 - p.y ** 2 / y0 ** 2) / (np.pi * x0 * y0)),
                 linear=lambda p: 1j * (p.Dx ** 2),
                 observe=[lambda a, p: A(a), lambda a, p: A(a),
                          lambda a, p: X.Int(A(a) * (p.kx ** 2 + p.ky ** 2), p.dk, p),
                          lambda a, p: np.sqrt(X.Int(p.y ** 2 * A(a), p.dx, p) / X.Int(A(a), p.dx, p)),
                          lambda a, p: np.sqrt(X.Int(p.x ** 2 * A(a), p.dx, p) / X.Int(A(a), p.dx, p)),
                          lambda a, p: np.sqrt(X.Int(p.ky ** 2 * A(a), p.dk, p) / X.Int(A(a), p.dk, p))],
                 transforms=[0, [0, 1, 1], [0, 1, 1], 0, 0, [0, 1, 1]],
                 compare=[None, None, lambda p: 1 / (2 * x0 ** 2) + 1 / (2 * y0 ** 2),
                          lambda p: y0 / np.sqrt(2), None, lambda p: 1 / (np.sqrt(2) * y0)])]


def soliton_deriv_n():
    return [dict(dimensions=2, points=[101, 101], method="RK4", order=4, ranges=[10, 15],
                 initial=lambda v, p: sech(p.x),
                 observe=[lambda a, p: a * np.conj(a), lambda a, p: X.Int(abs(X.D1(a, 1, p)) ** 2, p)],
                 boundaries=[None, [-1, -1]], deriv=lambda a, w, p: 1j * a * (np.conj(a) * a),
                 linear=lambda p: 0.5j * (p.Dx ** 2 - 1))]


def soliton_deriv_s():
    # D2 finite differences inside the drift on a periodic lattice, then a second
    # sequence with twice the nonlinearity (Examples/SPDE_2D/SolitonDerivS.m:11-23)
    p = dict(dimensions=2, order=4, points=[101, 51], steps=10, initial=lambda v, p: sech(p.x),
             deriv=lambda a, w, p: 1j * a * (np.conj(a) * a) + 0.5j * (X.D2(a, 1, p) - a),
             observe=[lambda a, p: a * np.conj(a), lambda a, p: X.Int(abs(X.D1(a, 1, p)) ** 2, p)])
    p1 = dict(p, deriv=lambda a, w, p: 2 * 1j * a * (np.conj(a) * a) + 0.5j * (X.D2(a, 1, p) - a))
    return [p, p1]


def _heat_in(v, p):
    x = p.x
    return np.concatenate([4 * np.sin(x) + np.sin(2 * x), 5 + 4 * np.cos(x) + np.cos(2 * x),
                           4 * np.sin(x / 2) + np.sin(3 * x / 2), 4 * np.cos(x / 2) + np.cos(3 * x / 2),
                           2 + np.cos(2 * x / 1.02) + np.sin(4 * x / 1.02)], axis=0)


def boundaries2():
    e = np.exp
    cmp = [lambda p: 4 * np.sin(p.x) * e(-p.t) + np.sin(2 * p.x) * e(-4 * p.t),
           lambda p: 5 + 4 * np.cos(p.x) * e(-p.t) + np.cos(2 * p.x) * e(-4 * p.t),
           lambda p: 4 * np.sin(p.x / 2) * e(-p.t / 4) + np.sin(3 * p.x / 2) * e(-9 * p.t / 4),
           lambda p: 4 * np.cos(p.x / 2) * e(-p.t / 4) + np.cos(3 * p.x / 2) * e(-9 * p.t / 4),
           lambda p: 2 + np.cos(2 * p.x / 1.02) * e(-4 * p.t / 1.02 ** 2) + np.sin(4 * p.x / 1.02) * e(-16 * p.t / 1.02 ** 2)]
    obs = [(lambda i: (lambda a, p: a[i:i + 1]))(i) for i in range(5)]
    p = dict(dimensions=2, points=[51, 51], method="MP", order=0, fields=5, ranges=[4, np.pi], origins=[0, 0],
             initial=_heat_in, observe=obs, compare=cmp,
             boundaries=[None, [[1, 1], [-1, -1], [1, -1], [-1, 1], [0, 0]]], linear=lambda p: p.Dx ** 2)
    p1 = dict(p)
    p1.update(linear=None, deriv=lambda a, w, p: X.D2(a, 1, p), steps=80, transfer=lambda b, v, p: _heat_in(0, p))
    return [p, p1]


def _per(x, t):
    P = np.exp(1j * t) * (4 * (1 + 2j * t) / (1 + 4 * (t ** 2 + x ** 2)) - 1)
    dP = -8 * x * np.exp(1j * t) * (4 * (1 + 2j * t) / (1 + 4 * (t ** 2 + x ** 2)) ** 2)
    return P, dP


def peregrine():
    def bv(a, c, d, p):
        P, dP = _per(p.origins[1], p.t)
        return [[P, P], [dP, -dP], [P, -dP], [dP, P]]
    sol = lambda p: abs(_per(p.x, p.t)[0] ** 2)
    return [dict(dimensions=2, noises=1, fields=4, order=2, ranges=[10, 10], origins=[-5, -5], points=[51, 161],
                 method="MP", boundaries=[None, [[1, 1], [-1, -1], [1, -1], [-1, 1]]], boundfun=bv,
                 initial=lambda v, p: _per(p.x, p.origins[0])[0] + np.zeros((4, 1, 1)), compare=[sol] * 4,
                 observe=[(lambda i: (lambda a, p: a[i:i + 1]))(i) for i in range(4)],
                 output=[(lambda i: (lambda o, p: abs(o[i]) ** 2))(i) for i in range(4)], steps=20,
                 deriv=lambda a, w, p: 1j * a * (np.conj(a) * a), linear=lambda p: 0.5j * p.Dx ** 2)]


def gaussian_av4d():
    def g4(p):
        sig = 1 + (p.t / 10) ** 2
        r2 = p.rr[1] ** 2 + p.rr[2] ** 2 + p.rr[3] ** 2 + p.rr[4] ** 2
        return sig ** -2 * np.exp(-r2 / sig)
    I = lambda a, p: a * np.conj(a)
    return [dict(dimensions=5, noises=2, points=[7, 15, 15, 15, 15],
                 initial=lambda w, p: np.exp(-0.5 * (p.r[1] ** 2 + p.r[2] ** 2 + p.r[3] ** 2 + p.r[4] ** 2)),
                 observe=[I, lambda a, p: X.Ave(I(a, p), p), lambda a, p: X.Int(I(a, p), p), I,
                          lambda a, p: X.Ave(I(a, p), p), lambda a, p: X.Int(I(a, p), p.dk, p)],
                 linear=lambda p: 1j * 0.05 * (p.D[1] ** 2 + p.D[2] ** 2 + p.D[3] ** 2 + p.D[4] ** 2),
                 transforms=[0, 0, 0, [0, 1, 1, 1, 1], [0, 1, 1, 1, 1], [0, 1, 1, 1, 1]],
                 compare=[g4, None, None, lambda p: 1], axes=[None, None, None, [0, -1, -1, -1, -1]])]


def gaussian3d():
    def g3(p):
        sig = 1 + (p.t / 10) ** 2
        return sig ** -1.5 * np.exp(-p.t - (p.x ** 2 + p.y ** 2 + p.z ** 2) / sig)
    return [dict(noises=[0, 0], dimensions=4, initial=lambda w, p: np.exp(-(p.x ** 2 + p.y ** 2 + p.z ** 2) / 2),
                 observe=[lambda a, p: a * np.conj(a)],
                 linear=lambda p: -0.5 + 1j * 0.05 * (p.Dx ** 2 + p.Dy ** 2 + p.Dz ** 2), compare=[g3])]


DETERMINISTIC = {
    "Soliton": soliton, "Characteristic": characteristic, "SolitonAv": soliton_av,
    "GaussianAv2D": gaussian_av2d, "GaussianKinetic": gaussian_kinetic, "SolitonDerivS": soliton_deriv_s,
    "SolitonDerivN": soliton_deriv_n,
    "Boundaries2": boundaries2, "Peregrine": peregrine, "GaussianAv4D": gaussian_av4d, "Gaussian3D": gaussian3d,
}
