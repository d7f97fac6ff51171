"""End-to-end through the C++ host mirror: config.json -> PGM in -> denoised
PGM out with the reference's PSNR report (src/main.cpp:56-112)."""

import json
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def write_pgm(path, img):
    a = np.clip(np.round(img), 0, 255).astype(np.uint8)
    path.write_bytes(b"P5\n%d %d\n255\n" % (a.shape[1], a.shape[0]) + a.tobytes())


def read_pgm(path):
    data = path.read_bytes()
    parts = data.split(maxsplit=4)
    w, h = int(parts[1]), int(parts[2])
    return np.frombuffer(parts[4][: w * h], np.uint8).reshape(h, w).astype(np.float32)


def test_batch_denoise_pgm(ksvd, synth, tmp_path, torch_cuda):
    clean = synth.clean_image(128, 9)
    noisy = synth.add_gaussian(clean, 20.0, 9)
    (tmp_path / "in").mkdir()
    (tmp_path / "out").mkdir()
    write_pgm(tmp_path / "in" / "img.pgm", noisy)
    write_pgm(tmp_path / "in" / "ref.pgm", clean)
    cfg = {"inputFolder": str(tmp_path / "in"), "outputFolder": str(tmp_path / "out"),
           "globalParams": {"patchWidthDim": 8, "patchHeightDim": 8, "slidingWidth": 2, "slidingHeight": 2,
                            "atoms": 64, "ompIter": 5, "ksvdIter": 3, "B&W": True, "speckle": False,
                            "type": "CUDA_K_SM100A", "minOmpIterBatch": 0, "subImageWidthDim": 0,
                            "subImageHeightDim": 0, "noiseVariance": 400.0},
           "files": [{"name": "img.pgm", "ref": "ref.pgm"}, {"name": "missing.pgm"}]}
    (tmp_path / "config.json").write_text(json.dumps(cfg))
    fails = ksvd.run_batch(tmp_path / "config.json")
    assert fails == 1  # the missing file fails to load (status -1), the other succeeds
    out = read_pgm(tmp_path / "out" / "8_8_img.pgm")
    assert synth.psnr(clean, out) > synth.psnr(clean, np.clip(np.round(noisy), 0, 255)) + 1.0
    # the CLI binary prints the reference's report
    exe = ksvd.PKG_DIR / "ksvd_denoise"
    r = subprocess.run([str(exe), str(tmp_path / "config.json")], capture_output=True, text=True, timeout=300)
    assert "PSNR after" in r.stdout and "Image Loading Failed" in r.stdout
