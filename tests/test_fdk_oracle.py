"""CPU: analytic properties of the FDK filter oracle (the restatement of
mat_codes/filtering.m and ParkerWeight.m; the MATLAB code itself cannot run
here) and the equivalence the GPU filter rests on: the zero-padded FFT
convolution equals a direct linear convolution with the spatial kernel."""
import numpy as np
import pytest

from oracle import fdk


def test_ram_lak_response_is_a_ramp():
    L = 1024
    filt = fdk.filter_response("ram-lak", L)
    k = np.arange(1, L // 2 + 1)
    w = 2 * np.pi * k / L
    # 2 |DTFT(ramp_flat)| = |w| / pi for the discrete Ram-Lak kernel
    np.testing.assert_allclose(filt[k], w / np.pi, rtol=2e-2, atol=2e-4)
    assert filt[0] < 1e-3                            # the kernel sums to ~0
    np.testing.assert_allclose(filt[1:L // 2], filt[L - 1:L // 2:-1])   # even


@pytest.mark.parametrize("window", ["shepp-logan", "cosine", "hamming", "hann"])
def test_windows_attenuate(window):
    L = 512
    r = fdk.filter_response("ram-lak", L)
    f = fdk.filter_response(window, L)
    assert np.all(f[1:L // 2 + 1] <= r[1:L // 2 + 1] + 1e-12)
    np.testing.assert_allclose(f[1:4], r[1:4], rtol=1e-3)    # ~1 at low frequency


def test_fft_filter_equals_direct_convolution():
    """The GPU evaluates filtering.m's padded FFT product as a direct linear
    convolution with h = real(ifft(filter)); show the two agree."""
    rng = np.random.default_rng(0)
    nu, nv, n_proj = 100, 3, 2
    sino = rng.random((n_proj, nv, nu))
    out = fdk.fdk_filter(sino, 600.0, 300.0, 1.0, 1.0, window="shepp-logan")
    # rebuild: weights, then direct convolution with the spatial kernel
    L = max(64, 2 ** fdk.nextpow2(2 * nu))
    h = np.real(np.fft.ifft(fdk.filter_response("shepp-logan", L)))
    us = (np.arange(nu) + 0.5) - nu / 2
    vs = (np.arange(nv) + 0.5) - nv / 2
    uu, vv = np.meshgrid(us, vs)
    x = sino * (600.0 / np.sqrt(600.0 ** 2 + uu ** 2 + vv ** 2))[None]
    d = np.arange(nu)[:, None] - np.arange(nu)[None, :]
    T = h[d % L]
    direct = np.einsum("pvj,ij->pvi", x, T) * (1 / 2 / 1.0 * (2 * np.pi / n_proj) / 2 * (600.0 / 300.0))
    np.testing.assert_allclose(out, direct, rtol=1e-10, atol=1e-12)


def test_parker_weights_count_each_line_once():
    """Parker weights lie in [0, 1] and, per detector column, add up to one
    half turn of views (each line integral counted once)."""
    nu, du, DSD = 128, 2.0, 600.0
    us = (np.arange(nu) + 0.5) * du - nu * du / 2
    fan = 2 * np.degrees(np.arctan(us[-1] / DSD))
    dang = 0.5
    n = int(np.ceil((180 + fan) / dang)) + 1
    for direction in (1, -1):
        W = fdk.parker_weights(us, DSD, dang, n, direction)
        assert W.min() >= 0 and W.max() <= 1
        np.testing.assert_allclose(W.sum(axis=0) * dang, 180.0, rtol=1.5e-2)


def test_cosine_weight_is_one_on_axis():
    sino = np.ones((1, 2, 2))
    # the four cells sit at u, v = +-0.5: weight DSD / sqrt(DSD^2 + 0.5)
    L = max(64, 2 ** fdk.nextpow2(4))
    assert L == 64
    out = fdk.fdk_filter(sino, 1e9, 1e9, 1.0, 1.0)
    assert np.isfinite(out).all()


@pytest.mark.parametrize("direction,ok", [(1, True), (-1, False)])
def test_parker_direction_weights_conjugate_pairs_to_one(direction, ok):
    """The Parker direction of a scan whose angles increase is +1.

    With this geometry's convention the ray at view phi through fan angle g
    has its conjugate at view phi + 180 + 2 g (degrees) with fan angle -g.
    Fan angles of whole degrees and a 1-degree view step put every conjugate
    on a measured view (2 g whole views later), and an even view count keeps
    every pweight off the region boundaries of ParkerWeight.m (where its
    three cases leave a weight of 1).  With dir = +1 the weights of every
    redundant pair add to one; with dir = -1 they do not."""
    DSD = 1000.0
    g = np.arange(-5, 6)
    us = DSD * np.tan(np.deg2rad(g.astype(float)))
    n_proj = 192
    W = fdk.parker_weights(us, DSD, 1.0, n_proj, direction)
    errs = [W[i, j] + W[i + 180 + 2 * gj, len(g) - 1 - j] - 1
            for i in range(n_proj) for j, gj in enumerate(g) if 0 <= i + 180 + 2 * gj < n_proj]
    assert len(errs) > 100
    assert (np.abs(errs).max() < 1e-12) == ok


def test_parker_direction_of_geometry():
    import nefct_b200 as nb
    from nefct_b200 import ops
    up = nb.ConeBeam((8, 8, 8), np.linspace(0, 3.6, 10), 100.0, 200.0, 16, 1.0, 8, 1.0)
    down = nb.ConeBeam((8, 8, 8), np.linspace(0, -3.6, 10), 100.0, 200.0, 16, 1.0, 8, 1.0)
    assert ops.parker_direction(up) == 1 and ops.parker_direction(down) == -1
