"""The device's scattering functions evaluated through the C ABI, for
checking them one by one against the reference's: EvaluateBsdf / PdfBsdf /
SampleBsdf (src/shading/bsdf.cpp:17-310) and TabulatedBSSRDF's Sr /
Sample_Sr / Pdf_Sr / Pdf_Sp (src/shading/bssrdf.cpp:153-266). Each call runs
a CUDA kernel over host arrays with the path tracer's own device code and
returns host arrays."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .render import MATERIAL_DTYPE, BssrdfTable


def _material(material) -> np.ndarray:
    m = np.ascontiguousarray(np.asarray(material, MATERIAL_DTYPE).reshape(1))
    return m


def bsdf_eval(material, wo, wi, normal, seeds):
    """f = EvaluateBsdf(wo, wi, n, rng) (n, 3) and then pdf = PdfBsdf(wo, wi,
    n, rng) (n,), rng = Rng(seeds[i]) per row."""
    m = _material(material)
    q = np.ascontiguousarray(np.concatenate([wo, wi, normal], axis=1), np.float32)
    s = np.ascontiguousarray(seeds, np.uint64).reshape(-1)
    n = q.shape[0]
    f = np.empty((n, 3), np.float32)
    pdf = np.empty(n, np.float32)
    _lib.check(_lib.lib().yrc_bsdf_eval(_lib.ptr(m), _lib.ptr(q), _lib.ptr(s), n, _lib.ptr(f), _lib.ptr(pdf)))
    return f, pdf


def bsdf_sample(material, wo, normal, u, seeds) -> np.ndarray:
    """SampleBsdf(wo, n, u, rng) per row -> (n, 9): wi, weight, pdf, valid, specular."""
    m = _material(material)
    q = np.ascontiguousarray(np.concatenate([wo, normal, u], axis=1), np.float32)
    s = np.ascontiguousarray(seeds, np.uint64).reshape(-1)
    out = np.empty((q.shape[0], 9), np.float32)
    _lib.check(_lib.lib().yrc_bsdf_sample(_lib.ptr(m), _lib.ptr(q), _lib.ptr(s), q.shape[0], _lib.ptr(out)))
    return out


def _table(t: dict) -> BssrdfTable:
    return BssrdfTable(len(t["rho_samples"]), len(t["radius_samples"]), _lib.ptr(t["rho_samples"]),
                       _lib.ptr(t["radius_samples"]), _lib.ptr(t["profile"]), _lib.ptr(t["rho_eff"]),
                       _lib.ptr(t["profile_cdf"]))


def bssrdf_eval(table: dict, sigma_a, sigma_s, eta: float, channels, u, r):
    """(Sample_Sr(ch, u), Pdf_Sr(ch, r), Sr(r)) of TabulatedBSSRDF(sigma_a,
    sigma_s, eta, table) per row; `table` is a build_bssrdf_table() dict."""
    ch = np.ascontiguousarray(channels, np.int32).reshape(-1)
    uu = np.ascontiguousarray(u, np.float32).reshape(-1)
    rr = np.ascontiguousarray(r, np.float32).reshape(-1)
    n = ch.size
    sa = np.ascontiguousarray(sigma_a, np.float32)
    ss = np.ascontiguousarray(sigma_s, np.float32)
    sample_r = np.empty(n, np.float32)
    pdf = np.empty(n, np.float32)
    sr = np.empty((n, 3), np.float32)
    tab = _table(table)
    _lib.check(_lib.lib().yrc_bssrdf_eval(C.byref(tab), _lib.ptr(sa), _lib.ptr(ss), float(eta), _lib.ptr(ch),
                                          _lib.ptr(uu), _lib.ptr(rr), n, _lib.ptr(sample_r), _lib.ptr(pdf),
                                          _lib.ptr(sr)))
    return sample_r, pdf, sr


def bssrdf_pdf_sp(table: dict, sigma_a, sigma_s, eta: float, queries) -> np.ndarray:
    """Pdf_Sp(po, ss, ts, ns, pi, ni) per row of 18 floats."""
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 18)
    sa = np.ascontiguousarray(sigma_a, np.float32)
    ss = np.ascontiguousarray(sigma_s, np.float32)
    out = np.empty(q.shape[0], np.float32)
    tab = _table(table)
    _lib.check(_lib.lib().yrc_bssrdf_pdf_sp(C.byref(tab), _lib.ptr(sa), _lib.ptr(ss), float(eta), _lib.ptr(q),
                                            q.shape[0], _lib.ptr(out)))
    return out
