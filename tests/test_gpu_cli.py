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


def write_ppm(path, rgb):
    a = np.clip(np.round(rgb), 0, 255).astype(np.uint8)
    path.write_bytes(b"P6\n%d %d\n255\n" % (a.shape[1], a.shape[0]) + a.tobytes())


def test_batch_denoise_colour_ppm(ksvd, synth, tmp_path, torch_cuda):
    """Colour input with B&W false (denoiser.cpp:47-51): the library denoises
    the luma channel 16 + (65.481 R + 128.553 G + 24.966 B) / 255 of the PPM,
    in the reference's orientation (the image transposed), and writes it
    min-max normalised to [0, 255] (denoiser.cpp:75).  The written PGM must
    equal that pipeline run through the Python binding, within one grey level
    (rounding at the normalisation)."""
    clean = synth.clean_image(96, 17)
    rgb = np.stack([clean, np.clip(0.7 * clean + 40.0, 0, 255), 255.0 - clean], axis=-1)
    noisy = np.clip(np.round(np.stack([synth.add_gaussian(rgb[..., c], 15.0, 17 + c) for c in range(3)],
                                      axis=-1)), 0, 255).astype(np.uint8)
    (tmp_path / "in").mkdir()
    (tmp_path / "out").mkdir()
    write_ppm(tmp_path / "in" / "col.ppm", noisy)
    gp = {"patchWidthDim": 8, "patchHeightDim": 8, "slidingWidth": 2, "slidingHeight": 2, "atoms": 48,
          "ompIter": 4, "ksvdIter": 2, "B&W": False, "speckle": False, "type": "CUDA_K_SM100A", "minOmpIterBatch": 0,
          "subImageWidthDim": 0, "subImageHeightDim": 0, "noiseVariance": 225.0}
    cfg = {"inputFolder": str(tmp_path / "in"), "outputFolder": str(tmp_path / "out"), "globalParams": gp,
           "files": [{"name": "col.ppm"}]}
    (tmp_path / "config.json").write_text(json.dumps(cfg))
    assert ksvd.run_batch(tmp_path / "config.json") == 0
    got = read_pgm(tmp_path / "out" / "8_8_col.ppm")
    f = noisy.astype(np.float32)
    luma = (np.float32(65.481) * f[..., 0] + np.float32(128.553) * f[..., 1] + np.float32(24.966) * f[..., 2])
    luma = np.float32(16.0) + luma / np.float32(255.0)
    params = ksvd.make_params(patch_width_dim=8, patch_height_dim=8, sliding_width=2, sliding_height=2, atoms=48,
                              omp_iter=4, ksvd_iter=2)
    with ksvd.Context(params) as c:
        out, _ = c.denoise(np.ascontiguousarray(luma.T), 225.0)
    out = out.T
    lo, hi = out.min(), out.max()
    want = np.clip(np.round((out - lo) * np.float32(255.0 / (hi - lo))), 0, 255)
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1.0
    # and it is a denoised luma image, not a copy of one channel
    assert synth.psnr(want, got) > 40.0
