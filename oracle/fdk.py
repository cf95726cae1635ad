"""TEST INFRASTRUCTURE: numpy restatement of the reference's FDK filtering.

Follows mat_codes/filtering.m:1-90 and mat_codes/ParkerWeight.m:1-29 of
bill52547/CT-NEF step by step in float64: cosine weight, optional Parker
weight, zero padding to max(64, 2^nextpow2(2 nu)), FFT, multiplication by
the windowed 2|FFT(ramp_flat)|, inverse FFT, crop and scale.  The MATLAB
code cannot run here (no MATLAB/Octave) and the reference holds no golden
vectors for it: parity unpinned.  This restatement is the FDK filter oracle;
it is checked against analytic properties of the filter
(tests/test_fdk_oracle.py), not against the reference run.

Array layout here is the GPU sinogram layout [nv][nb][na] (u = column a
fastest); the MATLAB code holds proj(u, v, view).
"""
from __future__ import annotations

import numpy as np


def nextpow2(n: int) -> int:
    p = 0
    while (1 << p) < n:
        p += 1
    return p


def ramp_flat(n: int) -> np.ndarray:
    """filtering.m:54-60."""
    nn = np.arange(-(n // 2), n // 2)
    h = np.zeros(n)
    h[n // 2] = 0.25
    odd = (nn % 2) == 1
    h[odd] = -1.0 / (np.pi * nn[odd]) ** 2
    return h


def filter_response(window: str, order: int, d: float = 1.0) -> np.ndarray:
    """filtering.m:63-88 (Filter)."""
    f_kernel = np.abs(np.fft.fft(ramp_flat(order))) * 2
    filt = f_kernel[: order // 2 + 1].copy()
    w = 2 * np.pi * np.arange(filt.size) / order
    win = window.lower()
    if win == "ram-lak":
        pass
    elif win == "shepp-logan":
        filt[1:] *= np.sin(w[1:] / (2 * d)) / (w[1:] / (2 * d))
    elif win == "cosine":
        filt[1:] *= np.cos(w[1:] / (2 * d))
    elif win == "hamming":
        filt[1:] *= 0.54 + 0.46 * np.cos(w[1:] / d)
    elif win == "hann":
        filt[1:] *= (1 + np.cos(w[1:] / d)) / 2
    else:
        raise ValueError(f"Invalid filter selected: {window}")
    filt[w > np.pi * d] = 0
    return np.concatenate([filt, filt[-2:0:-1]])


def parker_weights(us: np.ndarray, DSD: float, dang: float, n_proj: int, direction: int) -> np.ndarray:
    """ParkerWeight.m:5-27: weights [n_proj][nu] (degrees as in the MATLAB)."""
    a = np.arctan(us / DSD) / np.pi * 180
    fanang = abs(a[-1] - a[0]) / 2
    W = np.ones((n_proj, us.size))
    for i in range(1, n_proj + 1):
        pw = ((180 / dang - n_proj) / 2 + i) / (180 / dang) * 180 + direction * a
        w = W[i - 1]
        idx = (pw <= fanang / 2) & (pw > -fanang / 2)
        w[idx] *= np.maximum(np.sin(np.pi / 2 * (fanang / 2 + pw[idx]) / fanang), 0) ** 2
        idx = (pw >= 180 - fanang / 2) & (pw < 180 + fanang / 2)
        w[idx] *= np.maximum(np.cos(np.pi / 2 * (fanang / 2 + pw[idx] - 180) / fanang), 0) ** 2
        idx = (pw < -fanang / 2) | (pw > 180 + fanang / 2)
        w[idx] = 0
    return W


def fdk_filter(sino: np.ndarray, DSD: float, DSO: float, du: float, dv: float, *, a_shift=0.5, b_shift=0.5,
               window: str = "ram-lak", parker: int = 0, angles=None) -> np.ndarray:
    """filtering.m:1-52 on a [nv][nb][na] sinogram, float64 result."""
    n_proj, nv, nu = sino.shape
    us = (np.arange(nu) + a_shift) * du - nu * du / 2
    vs = (np.arange(nv) + b_shift) * dv - nv * dv / 2
    uu, vv = np.meshgrid(us, vs)                  # [nv][nu]
    w = DSD / np.sqrt(DSD ** 2 + uu ** 2 + vv ** 2)
    proj = sino.astype(np.float64) * w[None]
    if parker:
        dang = abs(float(angles[1]) - float(angles[0])) * 180 / np.pi
        proj = proj * parker_weights(us, DSD, dang, n_proj, parker)[:, None, :]
    filt_len = max(64, 2 ** nextpow2(2 * nu))
    filt = filter_response(window, filt_len)
    fproj = np.zeros((n_proj, nv, filt_len))
    lo = filt_len // 2 - nu // 2
    fproj[:, :, lo:lo + nu] = proj
    fproj = np.real(np.fft.ifft(np.fft.fft(fproj, axis=-1) * filt, axis=-1))
    out = fproj[:, :, lo:lo + nu]
    if parker:
        dang = abs(float(angles[1]) - float(angles[0])) * 180 / np.pi
        scale = 1 / 2 / du * (2 * np.pi / (180 / dang)) / 2 * (DSD / DSO)
    else:
        scale = 1 / 2 / du * (2 * np.pi / n_proj) / 2 * (DSD / DSO)
    return out * scale
