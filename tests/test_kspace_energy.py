"""The energy's gradient term as a k-space sum (CPU, numpy).

ENERGYC2's gradient term (misfit_uniform_time_seed_fftw_early.cpp:877-925 and 1043-1092,
grao2 taken twice at :915) is alpha * sum_x (gx^2 + 2 gy^2).  The reference forms gx and gy
as the real parts of complex inverse FFTs of -i k C^ over the full spectrum, with k at a
Nyquist index taken positive.  The mixed path's checkpoint column kernel sums the same
quantity in k-space over its half spectrum: weight 1 on the self-conjugate columns, 2 on
the others, and no derivative along an axis at that axis's Nyquist index (the real part of
the inverse transform cancels it).  These tests pin that identity on random fields.
"""
import numpy as np


def kvec(n, dx=0.125):
    """The reference's k-vector of one axis: 2 pi s(i) / (n dx), s(i) = i up to n/2 (the
    Nyquist index positive), i - n above."""
    s = np.arange(n)
    s = np.where(s <= n // 2, s, s - n)
    return 2.0 * np.pi * s / (n * dx)


def grad_energy_real_space(c, dx=0.125):
    """sum_x (gx^2 + 2 gy^2), gx = Re IFFT(-i kx C^) along axis 0, gy along axis 1."""
    C = np.fft.fftn(c)
    shape = c.shape
    kx = kvec(shape[0], dx).reshape((-1,) + (1,) * (c.ndim - 1))
    ky = kvec(shape[1], dx).reshape((1, -1) + (1,) * (c.ndim - 2))
    gx = np.fft.ifftn(-1j * kx * C).real
    gy = np.fft.ifftn(-1j * ky * C).real
    return float(np.sum(gx * gx + 2.0 * gy * gy))


def grad_energy_k_space(c, half_axis, dx=0.125):
    """The column kernel's sum: over the half spectrum along `half_axis` (m in 2-D, n in 3-D),
    sum_k w (kx^2 + 2 ky^2) |C^|^2 / P with kx = 0 at l = L/2 and ky = 0 at m = M/2."""
    C = np.fft.rfftn(np.moveaxis(c, half_axis, -1))
    C = np.moveaxis(C, -1, half_axis)
    shape = c.shape
    P = c.size
    kx = kvec(shape[0], dx)
    kx[shape[0] // 2] = 0.0
    ky = kvec(shape[1], dx)
    ky[shape[1] // 2] = 0.0
    nh = C.shape[half_axis]
    w = np.full(nh, 2.0)
    w[0] = 1.0
    w[-1] = 1.0  # the Nyquist column (even lengths)
    wshape = [1] * c.ndim
    wshape[half_axis] = nh
    if half_axis == 1:  # 2-D: ky runs along the half axis
        ky = ky[:nh]
    k2 = kx.reshape((-1,) + (1,) * (c.ndim - 1)) ** 2 + 2.0 * ky.reshape((1, -1) + (1,) * (c.ndim - 2)) ** 2
    return float(np.sum(w.reshape(wshape) * k2 * np.abs(C) ** 2) / P)


def test_kspace_gradient_term_2d():
    rng = np.random.default_rng(3)
    for L, M in ((64, 64), (32, 128), (128, 32)):
        c = 0.5 + 0.2 * rng.uniform(-1.0, 1.0, (L, M))
        real = grad_energy_real_space(c)
        ks = grad_energy_k_space(c, half_axis=1)
        assert abs(real - ks) <= 1e-11 * abs(real), (L, M, real, ks)


def test_kspace_gradient_term_3d():
    rng = np.random.default_rng(4)
    for L, M, N in ((32, 32, 8), (16, 32, 16)):
        c = 0.5 + 0.2 * rng.uniform(-1.0, 1.0, (L, M, N))
        real = grad_energy_real_space(c)
        ks = grad_energy_k_space(c, half_axis=2)
        assert abs(real - ks) <= 1e-11 * abs(real), (L, M, N, real, ks)


def test_nyquist_derivative_matters():
    """Keeping the derivative at the Nyquist indices (kx = kx(L/2) there) would overstate the
    term on a random field by far more than the tolerance above."""
    rng = np.random.default_rng(5)
    c = 0.5 + 0.2 * rng.uniform(-1.0, 1.0, (64, 64))
    real = grad_energy_real_space(c)
    C = np.fft.rfft(c, axis=1)
    kx = kvec(64)
    ky = kvec(64)[:33]
    w = np.full(33, 2.0)
    w[0] = w[-1] = 1.0
    naive = float(np.sum(w * (kx[:, None] ** 2 + 2.0 * ky[None, :] ** 2) * np.abs(C) ** 2) / c.size)
    assert abs(naive - real) > 1e-3 * abs(real)
