"""Seeded event-by-event initial conditions.

glauber_event() builds the Pb+Pb energy density used for the single-event
workloads: nucleons of each nucleus sampled from a Woods-Saxon density
(R = 6.62 fm, a = 0.546 fm), the nuclei offset by +-b/2 along x, a nucleon
is a participant when a nucleon of the other nucleus passes within
d^2 < sigma_NN/pi (sigma_NN = 6.4 fm^2 = 64 mb), each participant deposits a
Gaussian hotspot of width 0.5 fm with a Gamma(k=1.6, theta=1/1.6) weight, and
the transverse profile is multiplied by the longitudinal plateau
H(eta) = 1 for |eta| <= 2.0, exp(-(|eta|-2)^2 / (2*1.5^2)) beyond (the
plateau-with-Gaussian-tails form of kernel_glauber.cl:40-46), then scaled to
the requested peak energy density. Cell coordinates are those of
kernel_glauber.cl:86-98: x = (i - NX/2)*DX with integer division.
The random stream is numpy.random.default_rng(seed).
"""
import numpy as np


def woods_saxon_nucleons(rng, A=208, R=6.62, a=0.546):
    """A nucleon positions (A, 3) drawn from r^2 / (1 + exp((r-R)/a))."""
    rmax = R + 10.0 * a
    fmax = rmax * rmax
    out = np.empty((0,), np.float64)
    while out.size < A:
        r = rng.uniform(0.0, rmax, 4 * A)
        u = rng.uniform(0.0, fmax, 4 * A)
        keep = u < r * r / (1.0 + np.exp((r - R) / a))
        out = np.concatenate([out, r[keep]])
    r = out[:A]
    cost = rng.uniform(-1.0, 1.0, A)
    phi = rng.uniform(0.0, 2.0 * np.pi, A)
    sint = np.sqrt(1.0 - cost * cost)
    return np.stack([r * sint * np.cos(phi), r * sint * np.sin(phi), r * cost], axis=1)


def participants(rng, b, A=208, R=6.62, a=0.546, sigma_nn=6.4):
    """Transverse positions (n, 2) of the participants at impact parameter b."""
    na = woods_saxon_nucleons(rng, A, R, a)[:, :2] + np.array([0.5 * b, 0.0])
    nb = woods_saxon_nucleons(rng, A, R, a)[:, :2] - np.array([0.5 * b, 0.0])
    d2 = ((na[:, None, :] - nb[None, :, :]) ** 2).sum(-1)
    hit = d2 < sigma_nn / np.pi
    return np.concatenate([na[hit.any(1)], nb[hit.any(0)]])


def hotspots(rng, b, gamma_k=1.6, **kw):
    """Participant positions (n, 2) and their Gamma(k, 1/k) weights (n,)."""
    parts = participants(rng, b, **kw)
    w = rng.gamma(gamma_k, 1.0 / gamma_k, len(parts))
    return parts, w


def hotspot_table(b=8.0, seed=5):
    """(n, 3) float64 array of participant (x, y, weight) of the seeded event
    glauber_event(..., b, seed) builds, for the device generator
    (clv_hotspot_ini)."""
    parts, w = hotspots(np.random.default_rng(seed), b)
    return np.ascontiguousarray(np.column_stack([parts, w]), dtype=np.float64)


def transverse_profile(rng, nx, ny, dx, dy, b, width=0.5, gamma_k=1.6, **kw):
    """Sum of weighted Gaussian hotspots on the (nx, ny) grid (unnormalised)."""
    parts, w = hotspots(rng, b, gamma_k, **kw)
    x = (np.arange(nx) - nx // 2) * dx
    y = (np.arange(ny) - ny // 2) * dy
    ed = np.zeros((nx, ny))
    inv = 1.0 / (2.0 * width * width)
    for (px, py), wp in zip(parts, w):
        gx = np.exp(-(x - px) ** 2 * inv)
        gy = np.exp(-(y - py) ** 2 * inv)
        ed += wp * np.outer(gx, gy)
    return ed, len(parts)


def eta_profile(nz, dz, plateau=2.0, sigma=1.5):
    eta = (np.arange(nz) - nz // 2) * dz
    h = np.ones(nz)
    out = np.abs(eta) > plateau
    h[out] = np.exp(-(np.abs(eta[out]) - plateau) ** 2 / (2.0 * sigma * sigma))
    return h


def glauber_event(nx, ny, nz, dx, dy, dz, b=8.0, seed=5, edmax=50.0, dtype=np.float32):
    """(nx*ny*nz, 4) array of (ed, vx, vy, veta) with zero initial flow."""
    rng = np.random.default_rng(seed)
    exy, npart = transverse_profile(rng, nx, ny, dx, dy, b)
    h = eta_profile(nz, dz)
    ed = exy[:, :, None] * h[None, None, :]
    ed *= edmax / ed.max()
    out = np.zeros((nx * ny * nz, 4), dtype)
    out[:, 0] = ed.reshape(-1)
    return out


def gaussian_2d(nx, ny, dx, dy, e0=30.0, sx=2.0, sy=2.5, dtype=np.float64):
    """e0 * exp(-x^2/(2 sx^2) - y^2/(2 sy^2)), zero flow, NZ = 1."""
    x = (np.arange(nx) - nx // 2) * dx
    y = (np.arange(ny) - ny // 2) * dy
    ed = e0 * np.exp(-x[:, None] ** 2 / (2 * sx * sx) - y[None, :] ** 2 / (2 * sy * sy))
    out = np.zeros((nx * ny, 4), dtype)
    out[:, 0] = ed.reshape(-1)
    return out


def hotspot_ini(lib, params, ev, table, dx, dy, dz, width=0.5, plateau=2.0, sigma=1.5, edmax=50.0, stream=None):
    """glauber_event's energy density computed on the device into the SoA
    planes `ev` (a torch tensor of 4 planes described by `params`), from the
    host-sampled participant table of hotspot_table()."""
    import ctypes
    import torch
    from . import _lib
    dev = ev.device
    parts = torch.from_numpy(np.ascontiguousarray(table, dtype=np.float64)).to(dev)
    n = int(parts.shape[0])
    nbytes = int(lib.clv_hotspot_scratch_bytes(ctypes.byref(params), n))
    scratch = torch.empty(nbytes + 256, dtype=torch.uint8, device=dev)
    base = (scratch.data_ptr() + 255) // 256 * 256
    if stream is None:
        stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(lib.clv_hotspot_ini(ctypes.byref(params), ctypes.c_void_p(ev.data_ptr()),
                                   ctypes.c_void_p(parts.data_ptr()), n, float(dx), float(dy), float(dz), float(width),
                                   float(plateau), float(sigma), float(edmax), ctypes.c_void_p(base), nbytes, stream),
               'clv_hotspot_ini')
    return scratch, parts  # keep alive until the stream has run
