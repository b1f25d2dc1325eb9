"""Scene textures (RenderTexture, include/yaoray/scene/texture.hpp:37-51) and
device evaluation of their lookups through the C ABI: SampleTexture4
(src/shading/texture.cpp:297-309) and BuildTextureMipChain
(texture.cpp:242-264)."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib

# TextureFilter / TextureWrap (include/yaoray/scene/texture_options.hpp:7-17)
NEAREST, BILINEAR, TRILINEAR, EWA = 0, 1, 2, 3
REPEAT, CLAMP_TO_EDGE, MIRRORED_REPEAT = 0, 1, 2


class TextureStruct(C.Structure):
    """yrc_texture."""

    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("texels", C.c_void_p), ("filter", C.c_int32),
                ("wrap_s", C.c_int32), ("wrap_t", C.c_int32), ("reserved", C.c_int32)]


@dataclass
class Texture:
    """An RGBA32F image, (height, width, 4), row 0 first, with its filter and
    wrap modes. An empty array is a texture without data."""

    texels: np.ndarray
    filter: int = BILINEAR
    wrap_s: int = REPEAT
    wrap_t: int = REPEAT

    def c_struct(self) -> tuple[TextureStruct, np.ndarray]:
        """The yrc_texture and the array it points into (keep it alive)."""
        tx = np.ascontiguousarray(self.texels, np.float32)
        if tx.size == 0:
            return TextureStruct(0, 0, None, self.filter, self.wrap_s, self.wrap_t, 0), tx
        if tx.ndim != 3 or tx.shape[2] != 4:
            raise ValueError("texels must be (height, width, 4)")
        return TextureStruct(tx.shape[1], tx.shape[0], _lib.ptr(tx), self.filter, self.wrap_s, self.wrap_t, 0), tx


def textures_array(textures: list[Texture]):
    """A ctypes array of yrc_texture for `textures` and the arrays to keep."""
    arr = (TextureStruct * max(len(textures), 1))()
    keep = []
    for i, t in enumerate(textures):
        arr[i], tx = t.c_struct()
        keep.append(tx)
    return arr, keep


def sample(texture: Texture, uvs: np.ndarray, footprints: np.ndarray | None = None) -> np.ndarray:
    """SampleTexture4 on the device for (n, 2) uvs and optional (n, 4)
    footprints (dudx, dvdx, dudy, dvdy): (n, 4) RGBA."""
    ts, keep = texture.c_struct()
    uv = np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
    fp = None if footprints is None else np.ascontiguousarray(footprints, np.float32).reshape(-1, 4)
    if fp is not None and fp.shape[0] != uv.shape[0]:
        raise ValueError("one footprint per uv")
    out = np.empty((uv.shape[0], 4), np.float32)
    _lib.check(_lib.lib().yrc_texture_sample_eval(C.byref(ts), _lib.ptr(uv), _lib.ptr(fp), uv.shape[0],
                                                  _lib.ptr(out)))
    del keep
    return out


def mip_chain(texture: Texture) -> list[np.ndarray]:
    """Every level the device builds, the image first: (h, w, 4) arrays."""
    ts, keep = texture.c_struct()
    w, h = ts.width, ts.height
    cap, lw, lh = 0, w, h
    while w > 0 and h > 0:
        cap += lw * lh
        if lw == 1 and lh == 1:
            break
        lw, lh = max(1, (lw + 1) // 2), max(1, (lh + 1) // 2)
    out = np.empty(max(cap, 1) * 4, np.float32)
    dims = np.zeros(80, np.int32)
    count = C.c_int32(0)
    _lib.check(_lib.lib().yrc_texture_mip_chain_eval(C.byref(ts), _lib.ptr(out), cap, _lib.ptr(dims),
                                                     C.byref(count)))
    del keep
    levels, at = [], 0
    for k in range(count.value):
        lw, lh = int(dims[2 * k]), int(dims[2 * k + 1])
        levels.append(out[4 * at:4 * (at + lw * lh)].reshape(lh, lw, 4).copy())
        at += lw * lh
    return levels
