"""The fixed-point exact signs of insphere and orient3d (stream_b200/csrc/
exact_int.cuh, used by the exact stage for coordinates that are 0 or in
[2^-6, 2^18)), compiled for the host with g++ and checked against exact
rational arithmetic: random, co-spherical / co-planar lattice, 1-ulp
perturbed and extreme-magnitude inputs."""
import os
import shutil
import subprocess
from fractions import Fraction

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include "exact_int.cuh"
int main() {
    float p[5][3];
    while (true) {
        for (int i = 0; i < 5; ++i)
            for (int k = 0; k < 3; ++k)
                if (std::scanf("%a", &p[i][k]) != 1) return 0;
        const int s1 = sb::xint::insphere_sign(p[0], p[1], p[2], p[3], p[4]);
        const int s2 = sb::xint::orient3d_sign(p[0][0], p[0][1], p[0][2], p[1][0], p[1][1], p[1][2], p[2][0], p[2][1],
                                               p[2][2], p[3][0], p[3][1], p[3][2]);
        std::printf("%d %d\n", s1, s2);
    }
}
"""


def _sgn(x):
    return (x > 0) - (x < 0)


def _det3(m):
    return (m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0])
            + m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]))


def _insphere(p):
    e = p[4]
    rows = []
    for q in p[:4]:
        d = [q[k] - e[k] for k in range(3)]
        rows.append(d + [d[0] * d[0] + d[1] * d[1] + d[2] * d[2]])
    s = 0
    for k in range(4):
        minor = [[rows[r][c] for c in range(4) if c != k] for r in range(1, 4)]
        s += (-1) ** k * rows[0][k] * _det3(minor)
    return _sgn(s)


def _orient3d(p):
    d = p[3]
    return _sgn(_det3([[p[i][k] - d[k] for k in range(3)] for i in range(3)]))


def _cases():
    rng = np.random.default_rng(3)
    cube = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]], float)
    out = []
    for _ in range(300):
        out.append(0.05 + 0.9 * rng.random((5, 3)))
    for s in (3 / 99.0, 0.37, 1.0, 1000.0):
        for o in (0.0, 2 / 99.0, 0.5, 17.0):
            for _ in range(25):
                out.append(cube[rng.choice(8, 5, replace=False)] * s + o)  # co-spherical, often co-planar
    for _ in range(300):
        p = (cube[rng.choice(8, 5, replace=False)] * rng.choice([0.01, 0.1, 1 / 99.0]) + 0.05 + rng.random(3)).astype(
            np.float32)
        k = rng.integers(0, 5)
        p[k] = np.nextafter(p[k], np.float32(2.0))
        out.append(p.astype(float))
    for _ in range(100):  # extremes of the range
        q = rng.choice([0.015625, 0.02, 1.5, 262143.0, 131072.5], size=(5, 3)) * rng.choice([-1.0, 1.0], size=(5, 3))
        out.append(q)
    return np.array(out, np.float32)


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_fixed_point_signs_vs_rationals(tmp_path):
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = tmp_path / "drv"
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "stream_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    pts = _cases()
    assert np.all((pts == 0) | ((np.abs(pts) >= 2.0 ** -6) & (np.abs(pts) < 2.0 ** 18)))
    text = "\n".join(" ".join(float(v).hex() for v in q.reshape(-1)) for q in pts)
    r = subprocess.run([str(exe)], input=text, capture_output=True, text=True, check=True)
    got = np.array([[int(t) for t in ln.split()] for ln in r.stdout.splitlines()])
    assert got.shape == (len(pts), 2)
    want = np.array([[_insphere([[Fraction(float(v)) for v in q] for q in p]),
                      _orient3d([[Fraction(float(v)) for v in q] for q in p])] for p in pts])
    assert np.array_equal(got, want)
    assert (want[:, 0] == 0).sum() > 50 and (want[:, 1] == 0).sum() > 50  # the degenerate cases are exercised
