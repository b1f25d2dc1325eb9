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
