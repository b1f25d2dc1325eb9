"""Drop-in check: the reference's own PBRT frontend and CpuBackend, with
yr::CudaBackend implemented by integration/yaoray_cuda_backend.cpp linked in
place of the reference's CUDA stub (oracle/_ref/yaoray_dropin, built by
`make -C oracle dropin`), render the same Cornell file. The CUDA film must
carry bit-identical first-hit AOVs and sample counts and a beauty image within
the render-parity bound; the progress callback must run once per pass."""
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from yaoray_b200 import cornell
from yaoray_b200.render import FILM_PIXEL_DTYPE

pytestmark = pytest.mark.gpu
DRIVER = Path(__file__).resolve().parent.parent / "oracle" / "_ref" / "yaoray_dropin"


def test_reference_cli_path_with_cuda_backend(cuda, tmp_path):
    if not DRIVER.exists():
        pytest.skip("drop-in driver not built (needs the reference sources)")
    scene = tmp_path / "cornell.pbrt"
    scene.write_text(cornell.pbrt_text(80, 64, 32, 8))
    out = subprocess.run([str(DRIVER), str(scene), str(tmp_path / "r")], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    info = json.loads(out.stdout.strip().splitlines()[-1])
    cpu = np.fromfile(tmp_path / "r.cpu.film", FILM_PIXEL_DTYPE)
    gpu = np.fromfile(tmp_path / "r.cuda.film", FILM_PIXEL_DTYPE)
    assert cpu.size == gpu.size == 80 * 64
    assert np.array_equal(cpu["samples"], gpu["samples"])
    for k in ("albedo_sum", "normal_sum", "depth_sum", "aov_samples"):
        assert cpu[k].tobytes() == gpu[k].tobytes(), k
    c = cpu["sum"] / cpu["samples"][:, None]
    g = gpu["sum"] / gpu["samples"][:, None]
    assert abs(g.mean() / c.mean() - 1) < 0.01
    assert info["cuda_progress_calls"] == 32
    assert abs(info["cuda_rays"] / info["cpu_rays"] - 1) < 0.02


def test_reference_cli_path_textured_scene(cuda, tmp_path):
    """Image-map textures through the reference's own frontend (TGA loading,
    sRGB decoding, uvs from "point2 uv") and the drop-in adapter's texture
    and uv marshalling: the floor bilinear, the back wall with the
    frontend's default EWA filter."""
    if not DRIVER.exists():
        pytest.skip("drop-in driver not built (needs the reference sources)")
    rng = np.random.default_rng(4)
    y, x = np.mgrid[0:32, 0:32]
    checks = np.where((((x // 4) + (y // 4)) % 2 == 0)[..., None], [230, 220, 200], [40, 60, 120]).astype(np.uint8)
    cornell.write_tga(tmp_path / "floor.tga", checks)
    cornell.write_tga(tmp_path / "wall.tga", rng.integers(60, 250, (24, 40, 3)).astype(np.uint8))
    scene = tmp_path / "textured.pbrt"
    scene.write_text(cornell.pbrt_text_textured(80, 64, 32, 8, "floor.tga", "wall.tga"))
    out = subprocess.run([str(DRIVER), str(scene), str(tmp_path / "r")], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    cpu = np.fromfile(tmp_path / "r.cpu.film", FILM_PIXEL_DTYPE)
    gpu = np.fromfile(tmp_path / "r.cuda.film", FILM_PIXEL_DTYPE)
    assert np.array_equal(cpu["samples"], gpu["samples"])
    for k in ("normal_sum", "depth_sum", "aov_samples"):
        assert cpu[k].tobytes() == gpu[k].tobytes(), k
    a, b = gpu["albedo_sum"], cpu["albedo_sum"]
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
    assert np.mean(np.all(a.view(np.uint32) == b.view(np.uint32), axis=-1)) >= 0.99
    assert len(np.unique(b.round(3), axis=0)) > 50  # the textures are visible in the albedo
    c = cpu["sum"] / cpu["samples"][:, None]
    g = gpu["sum"] / gpu["samples"][:, None]
    assert abs(g.mean() / c.mean() - 1) < 0.01


def test_reference_cli_path_analytic_lights(cuda, tmp_path):
    """Point, spot and distant LightSources compiled by the reference's
    frontend and passed through the adapter (the library builds their power
    alias table), next to the box's area light."""
    if not DRIVER.exists():
        pytest.skip("drop-in driver not built (needs the reference sources)")
    lines = cornell.pbrt_text(80, 64, 32, 8).splitlines()
    world = lines.index("WorldBegin")
    lights = ['LightSource "point" "rgb I" [3 2.5 2] "point3 from" [1.2 4.5 2.0]',
              'LightSource "spot" "rgb I" [8 8 10] "point3 from" [4.0 5.0 3.5] "point3 to" [3.5 0 3.0] '
              '"float coneangle" [30] "float conedeltaangle" [8]',
              'LightSource "distant" "rgb L" [0.4 0.4 0.35] "point3 from" [0 0 0] "point3 to" [0.2 -1 0.6]']
    scene = tmp_path / "lights.pbrt"
    scene.write_text("\n".join(lines[:world + 1] + lights + lines[world + 1:]) + "\n")
    out = subprocess.run([str(DRIVER), str(scene), str(tmp_path / "r")], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    info = json.loads(out.stdout.strip().splitlines()[-1])
    cpu = np.fromfile(tmp_path / "r.cpu.film", FILM_PIXEL_DTYPE)
    gpu = np.fromfile(tmp_path / "r.cuda.film", FILM_PIXEL_DTYPE)
    assert np.array_equal(cpu["samples"], gpu["samples"])
    for k in ("albedo_sum", "normal_sum", "depth_sum", "aov_samples"):
        assert cpu[k].tobytes() == gpu[k].tobytes(), k
    c = cpu["sum"] / cpu["samples"][:, None]
    g = gpu["sum"] / gpu["samples"][:, None]
    assert abs(g.mean() / c.mean() - 1) < 0.01
    assert abs(info["cuda_rays"] / info["cpu_rays"] - 1) < 0.02


def test_reference_cli_path_measured_material(cuda, tmp_path):
    """A measured material read by the reference's loader from an RGL
    tensor file (the seeded synthetic BRDF written by
    measured.write_tensor_file) on both boxes, passed through the adapter's
    measured-BRDF marshalling."""
    if not DRIVER.exists():
        pytest.skip("drop-in driver not built (needs the reference sources)")
    from yaoray_b200 import measured

    measured.write_tensor_file(tmp_path / "synthetic.bsdf", measured.synthetic_brdf(3))
    lines = cornell.pbrt_text(80, 64, 32, 8).splitlines()
    world = lines.index("WorldBegin")
    out_lines = lines[:world + 1] + ['MakeNamedMaterial "meas" "string type" ["measured"] '
                                     '"string filename" ["synthetic.bsdf"]']
    shape = 0
    for line in lines[world + 1:]:
        if line.startswith('NamedMaterial "white"') and shape in (5, 6):
            line = 'NamedMaterial "meas"'
        if line.startswith('Shape "trianglemesh"'):
            shape += 1
        out_lines.append(line)
    scene = tmp_path / "measured.pbrt"
    scene.write_text("\n".join(out_lines) + "\n")
    out = subprocess.run([str(DRIVER), str(scene), str(tmp_path / "r")], capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stderr
    cpu = np.fromfile(tmp_path / "r.cpu.film", FILM_PIXEL_DTYPE)
    gpu = np.fromfile(tmp_path / "r.cuda.film", FILM_PIXEL_DTYPE)
    for k in ("normal_sum", "depth_sum", "aov_samples"):
        assert cpu[k].tobytes() == gpu[k].tobytes(), k
    c = cpu["sum"] / cpu["samples"][:, None]
    g = gpu["sum"] / gpu["samples"][:, None]
    assert abs(g.mean() / c.mean() - 1) < 0.01
