"""Coefficients of the degree-5 polynomial for 2^f, |f| <= 1/2, used by vexp
(vgr_common.cuh) and by the oracle's vo_exp.

The Remez exchange algorithm on [-1/2, 1/2] for the relative error
|p(f) / 2^f - 1|, solved in float64 from Chebyshev extrema; the printed
coefficients are the float32 roundings compiled into both files (equi-
oscillation error 7.5e-8 before rounding; the float32 evaluation with a
two-step Cody-Waite reduction stays within 2.3e-7 relative of exp on
[-87, 88]).

Usage: python exp2_minimax.py
"""

from __future__ import annotations

import numpy as np


def remez(degree: int, iterations: int = 30) -> tuple[np.ndarray, float]:
    a, b = -0.5, 0.5
    k = np.arange(degree + 2)
    x = np.cos(np.pi * k / (degree + 1))[::-1] * (b - a) / 2 + (a + b) / 2
    grid = np.linspace(a, b, 200_001)
    for _ in range(iterations):
        # p(x_i) - 2^x_i = (-1)^i E 2^x_i at the reference points.
        system = np.zeros((degree + 2, degree + 2))
        for i, xi in enumerate(x):
            system[i, : degree + 1] = xi ** np.arange(degree + 1)
            system[i, degree + 1] = -((-1) ** i) * 2.0**xi
        solution = np.linalg.solve(system, 2.0**x)
        coeffs = solution[: degree + 1]
        err = np.polyval(coeffs[::-1], grid) / 2.0**grid - 1.0
        # New reference: the extremum of each sign-constant segment.
        signs = np.sign(err)
        cuts = np.nonzero(signs[1:] != signs[:-1])[0] + 1
        segments = np.split(np.arange(grid.size), cuts)
        points = [seg[np.argmax(np.abs(err[seg]))] for seg in segments]
        if len(points) != degree + 2:
            points = sorted(sorted(points, key=lambda p: -abs(err[p]))[: degree + 2])
        x = grid[points]
    return coeffs, float(np.max(np.abs(err)))


if __name__ == "__main__":
    coeffs, error = remez(5)
    print(f"max relative error {error:.3e}")
    for k, c in enumerate(coeffs):
        print(f"c{k} = {float(np.float32(c)):.9e}f")
