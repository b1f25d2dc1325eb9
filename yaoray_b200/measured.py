"""Measured (RGL) BRDFs (MeasuredBrdf, include/yaoray/shading/measured_brdf.hpp)
as plain arrays for the C ABI, device evaluation / sampling for checking,
and a seeded synthetic BRDF with the tensor shapes of an isotropic RGL file
(the RGL data files themselves are not part of this project)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib


class MeasuredStruct(C.Structure):
    """yrc_measured_brdf."""

    _fields_ = [("n_theta_i", C.c_int32), ("n_phi_i", C.c_int32), ("n_wavelengths", C.c_int32),
                ("ndf_rows", C.c_int32), ("ndf_cols", C.c_int32), ("vndf_rows", C.c_int32),
                ("vndf_cols", C.c_int32), ("res", C.c_int32)] + \
        [(k, C.c_void_p) for k in ("theta_i", "phi_i", "wavelengths", "ndf", "sigma", "vndf", "luminance",
                                   "spectra")]


@dataclass
class MeasuredBrdf:
    theta_i: np.ndarray      # (n_theta_i,)
    phi_i: np.ndarray        # (n_phi_i,), at most 2 (isotropic)
    wavelengths: np.ndarray  # (n_wl,)
    ndf: np.ndarray          # (rows, cols)
    sigma: np.ndarray        # (rows, cols)
    vndf: np.ndarray         # (n_phi_i, n_theta_i, vrows, vcols)
    luminance: np.ndarray    # (n_phi_i, n_theta_i, res, res)
    spectra: np.ndarray      # (n_phi_i, n_theta_i, n_wl, res, res)

    def c_struct(self) -> tuple[MeasuredStruct, list]:
        arrs = {k: np.ascontiguousarray(getattr(self, k), np.float32)
                for k in ("theta_i", "phi_i", "wavelengths", "ndf", "sigma", "vndf", "luminance", "spectra")}
        s = MeasuredStruct(arrs["theta_i"].size, arrs["phi_i"].size, arrs["wavelengths"].size,
                           arrs["ndf"].shape[0], arrs["ndf"].shape[1], arrs["vndf"].shape[2], arrs["vndf"].shape[3],
                           arrs["luminance"].shape[2], *[_lib.ptr(arrs[k]) for k in
                                                          ("theta_i", "phi_i", "wavelengths", "ndf", "sigma", "vndf",
                                                           "luminance", "spectra")])
        return s, list(arrs.values())


def measured_array(brdfs: list[MeasuredBrdf]):
    arr = (MeasuredStruct * max(len(brdfs), 1))()
    keep = []
    for i, b in enumerate(brdfs):
        arr[i], k = b.c_struct()
        keep.append(k)
    return arr, keep


def evaluate(brdf: MeasuredBrdf, wo, wi, n) -> tuple[np.ndarray, np.ndarray]:
    """EvaluateMeasured and PdfMeasured on the device: (f (n, 3), pdf (n,))."""
    q = np.ascontiguousarray(np.concatenate([np.reshape(wo, (-1, 3)), np.reshape(wi, (-1, 3)),
                                             np.reshape(n, (-1, 3))], 1), np.float32)
    f = np.empty((q.shape[0], 3), np.float32)
    pdf = np.empty(q.shape[0], np.float32)
    s, keep = brdf.c_struct()
    _lib.check(_lib.lib().yrc_measured_eval(C.byref(s), _lib.ptr(q), q.shape[0], _lib.ptr(f), _lib.ptr(pdf)))
    del keep
    return f, pdf


def sample(brdf: MeasuredBrdf, wo, n, u) -> np.ndarray:
    """SampleMeasured on the device: (n, 8) rows of wi, weight, pdf, valid."""
    q = np.ascontiguousarray(np.concatenate([np.reshape(wo, (-1, 3)), np.reshape(n, (-1, 3)),
                                             np.reshape(u, (-1, 2))], 1), np.float32)
    out = np.empty((q.shape[0], 8), np.float32)
    s, keep = brdf.c_struct()
    _lib.check(_lib.lib().yrc_measured_sample(C.byref(s), _lib.ptr(q), q.shape[0], _lib.ptr(out)))
    del keep
    return out


def synthetic_brdf(seed: int = 0, n_theta_i: int = 6, res: int = 16, wavelengths=(400, 460, 520, 580, 640, 700)):
    """A seeded isotropic BRDF with RGL tensor shapes: a rough-glossy NDF
    (theta_m x phi_m), smooth positive sigma / vndf / luminance slices per
    incident angle and per-wavelength spectra that tint it."""
    rng = np.random.default_rng(seed)
    th = np.linspace(0.0, 1.45, n_theta_i).astype(np.float32)
    phi = np.array([0.0], np.float32)
    wl = np.asarray(wavelengths, np.float32)
    y, x = np.mgrid[0:res, 0:res] / (res - 1.0)
    ndf = (np.exp(-(y / 0.35) ** 2) * (1.0 + 0.2 * np.cos(2 * np.pi * x)) + 0.02).astype(np.float32)
    sigma = (0.8 + 0.4 * y + 0.05 * rng.random((res, res))).astype(np.float32)
    vndf = np.empty((1, n_theta_i, res, res), np.float32)
    lum = np.empty((1, n_theta_i, res, res), np.float32)
    spec = np.empty((1, n_theta_i, wl.size, res, res), np.float32)
    for k in range(n_theta_i):
        vndf[0, k] = np.exp(-((y - 0.1 * k / n_theta_i) / 0.4) ** 2) + 0.05 + 0.05 * rng.random((res, res))
        lum[0, k] = np.exp(-(y / (0.5 + 0.1 * k)) ** 2) * (1.0 + 0.3 * x) + 0.03
        for j, w in enumerate(wl):
            tint = 0.3 + 0.6 * np.exp(-((w - 600.0) / 120.0) ** 2)
            spec[0, k, j] = lum[0, k] * tint * (1.0 + 0.1 * rng.random((res, res)))
    return MeasuredBrdf(th, phi, wl, ndf, sigma, vndf, lum, spec)


def write_tensor_file(path, brdf: MeasuredBrdf) -> None:
    """Saves `brdf` as an RGL .bsdf file in the Mitsuba tensor-file layout
    (the format the reference's LoadMeasuredBrdf reads): magic
    "tensor_file\\0", version 1.0, the field count, then per field its name,
    rank, dtype (10 = float32), absolute data offset and shape, followed by
    the little-endian data."""
    import struct

    fields = [(k, np.ascontiguousarray(getattr(brdf, k), np.float32))
              for k in ("theta_i", "phi_i", "wavelengths", "ndf", "sigma", "vndf", "luminance", "spectra")]
    header = b"tensor_file\0" + bytes([1, 0]) + struct.pack("<I", len(fields))
    size = len(header) + sum(2 + len(k) + 2 + 1 + 8 + 8 * a.ndim for k, a in fields)
    descs, blobs, offset = b"", b"", size
    for k, a in fields:
        descs += struct.pack("<H", len(k)) + k.encode() + struct.pack("<HBQ", a.ndim, 10, offset)
        descs += b"".join(struct.pack("<Q", d) for d in a.shape)
        blobs += a.tobytes()
        offset += a.nbytes
    with open(path, "wb") as f:
        f.write(header + descs + blobs)
