"""Coefficients of the FP64 logarithm of the fused kernels (pf_log in
pf3d_device.cuh) and their error.

log x = k ln2 + 2s + 2s z P(z) with s = (m-1)/(m+1), m in [sqrt(1/2), sqrt(2)),
z = s^2 <= 0.029438.  P(z) = (atanh(sqrt z)/sqrt z - 1)/z (the Taylor series of
atanh: 1/3 + z/5 + z^2/7 + ...) is replaced by its Chebyshev interpolant of
degree 6 on [0, 0.029441] (Lanczos economization; mpmath.chebyfit at 50
digits).  The coefficients are rounded to double and the error of the rounded
polynomial, evaluated exactly, is measured on a fine grid; 2s z P(z) carries
it into log x multiplied by at most z.

    python log_coeffs.py
"""
import mpmath as mp

mp.mp.dps = 50
S_MAX = mp.mpf("0.17157287525380996")          # (sqrt 2 - 1)/(sqrt 2 + 1), rounded up
Z_MAX = S_MAX ** 2 * mp.mpf("1.0001")


def P(z):
    if z == 0:
        return mp.mpf(1) / 3
    r = mp.sqrt(z)
    return (mp.atanh(r) / r - 1) / z


def coefficients(degree=6, grid=4000):
    """(coefficients highest degree first, max |P6 - P| on the grid)."""
    poly, _ = mp.chebyfit(P, [0, Z_MAX], degree + 1, error=True)
    coeffs = [float(c) for c in poly]          # Horner order
    worst = mp.mpf(0)
    for i in range(grid + 1):
        z = Z_MAX * i / grid
        v = mp.mpf(0)
        for c in coeffs:
            v = v * z + mp.mpf(c)
        worst = max(worst, abs(v - P(z)))
    return coeffs, float(worst)


def main():
    coeffs, worst = coefficients()
    for c in coeffs:
        print(repr(c))
    print("max |P6 - P| = %.3g, in log x at most %.3g" % (worst, worst * float(Z_MAX)))


if __name__ == "__main__":
    main()
