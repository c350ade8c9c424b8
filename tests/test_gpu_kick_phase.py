"""Direct accuracy test of the kick's sin / cos (qj_selftest_sincos).

The fused kick rotates psi by exp(-i theta), theta = (m / hbar)(dt / 2) V in
float64 (quantum-stars.py:300 takes exp(-1j V dt / 2) of the complex64 field).
The kernel reduces theta to r in [-pi/4, pi/4] in float64 (quadrant
n = rint(2 theta / pi), two-part pi / 2) and evaluates the Taylor series of
sin r and cos r to degree 9 / 10 in float32; below |theta| = 2^-10 it takes
sin ~ x (1 - x^2 / 6), cos ~ 1 - x^2 / 2 in float32 without reduction.
Checked here against float64 NumPy sin / cos (an independent reference) over a
sweep of theta: log-spaced magnitudes 1e-9 .. 1e3 of both signs, a dense band
around the 2^-10 switch, every multiple of pi / 4 up
to |theta| = 1000 with offsets of 0, 1e-12, 1e-7 and 1e-4 (the quadrant
boundaries), and uniform random values.

Bounds: absolute error <= 2 * 2^-24 (the rotation multiplies a unit-modulus
factor, so absolute error is what reaches psi), and <= 2 float32 ulp of the
value wherever |value| >= 2^-10.  A float32 evaluation of the same formulas
on the CPU reaches 1.39 * 2^-24 and 1.83 ulp.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def thetas():
    mag = np.concatenate([np.logspace(-9, 3, 300001), 2.0 ** -10 * (1 + np.linspace(-1e-6, 1e-6, 201))])
    k = np.arange(-1273, 1274)
    offs = np.array([0.0, 1e-12, -1e-12, 1e-7, -1e-7, 1e-4, -1e-4])
    near = (k[:, None] * (np.pi / 4) + offs[None, :]).ravel()
    rnd = np.random.default_rng(0).uniform(-1000.0, 1000.0, 200000)
    return np.concatenate([mag, -mag, near, rnd, [0.0]])


def test_kick_sincos_accuracy():
    import qj

    lib = qj.lib()
    th = thetas()
    d_th = torch.as_tensor(th, dtype=torch.float64, device="cuda")
    out = torch.empty((len(th), 2), dtype=torch.float32, device="cuda")
    rc = lib.qj_selftest_sincos(ctypes.c_void_p(d_th.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                len(th), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, lib.qj_last_error()
    got = out.cpu().numpy().astype(np.float64)
    for j, ref in ((0, np.sin(th)), (1, np.cos(th))):
        err = np.abs(got[:, j] - ref)
        assert err.max() <= 2.0 * 2.0 ** -24, (j, err.max(), th[np.argmax(err)])
        big = np.abs(ref) >= 2.0 ** -10
        ulp = np.spacing(np.abs(ref[big]).astype(np.float32)).astype(np.float64)
        assert (err[big] / ulp).max() <= 2.0, (j, (err[big] / ulp).max())
    # the pair stays on the unit circle to float32 rounding
    assert np.abs(np.hypot(got[:, 0], got[:, 1]) - 1.0).max() <= 4.0 * 2.0 ** -24


def test_kick_sincos_rejects_bad_arguments():
    import qj

    lib = qj.lib()
    assert lib.qj_selftest_sincos(None, None, 4, None) == qj._lib.QJ_ERR_ARG
    x = torch.zeros(2, dtype=torch.float64, device="cuda")
    assert lib.qj_selftest_sincos(ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()),
                                  -1, None) == qj._lib.QJ_ERR_ARG
