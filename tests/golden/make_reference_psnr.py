"""Makes tests/golden/reference_barbara_psnr.npz from the reference's own test
images (test/images of newfla/CUDA-K-SVD-Denoising, read from a local copy of
the reference; run where that copy exists).

Kept: the clean barbara image and its three noisy versions (noise variances
0.03, 0.05, 0.1 in the reference's file names) as uint8, and the PSNR against
the clean image of each of the reference's stored GPU outputs for 256 atoms
after 1, 5 and 10 K-SVD iterations (test/images/output/barbara/GPU/
8_8_barbara_<noise>_256_<iterations>.png).  The reference's src/config.json
gives their settings: 8 x 8 patches, stride 2, 256 atoms, 5 OMP atoms.
"""
import sys
from pathlib import Path

import numpy as np
from PIL import Image

if len(sys.argv) != 2:
    sys.exit("usage: make_reference_psnr.py <path of the reference project>")
REF = Path(sys.argv[1]) / "test" / "images"
OUT = Path(__file__).resolve().parent / "reference_barbara_psnr.npz"


def read(p):
    return np.asarray(Image.open(p).convert("L"), dtype=np.uint8)


def psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10.0 * np.log10(255.0 ** 2 / mse)


def main():
    clean = read(REF / "input" / "barbara_ref.png")
    levels = ["0,03", "0,05", "0,1"]
    iters = [1, 5, 10]
    noisy = np.stack([read(REF / "input" / f"barbara_{lv}.png") for lv in levels])
    ref_psnr = np.array([[psnr(clean, read(REF / "output" / "barbara" / "GPU" / f"8_8_barbara_{lv}_256_{it}.png"))
                          for it in iters] for lv in levels])
    np.savez_compressed(OUT, kind="reference_psnr", clean=clean, noisy=noisy, levels=np.array(levels),
                        iters=np.array(iters), ref_psnr=ref_psnr, patch=8, stride=2, atoms=256, omp_iter=5)
    print(OUT, OUT.stat().st_size, "bytes")
    print(np.round(ref_psnr, 2))


if __name__ == "__main__":
    main()
