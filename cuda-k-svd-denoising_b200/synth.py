"""Seeded synthetic grayscale test images.

The reference denoises image files (PNG/JPG via CImg).  Here the inputs are
synthetic: a sum of sinusoidal gratings (random orientation, period, phase and
amplitude) rescaled to [0, 255], with flat rectangles painted over it, then
additive Gaussian noise or multiplicative Gamma (speckle) noise.  Everything is
drawn from ``numpy.random.default_rng(seed)`` so a seed fixes the image.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def clean_image(size: int, seed: int, n_gratings: int = 12, n_rects: int = 40,
                period: tuple = (4.0, 64.0)) -> np.ndarray:
    """Square (size, size) float32 image with values in [0, 255]."""
    rng = np.random.default_rng(seed)
    yy = np.arange(size, dtype=np.float64)[:, None]
    xx = np.arange(size, dtype=np.float64)[None, :]
    img = np.zeros((size, size), np.float64)
    for _ in range(n_gratings):
        theta = rng.uniform(0.0, np.pi)
        per = rng.uniform(*period)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        amp = rng.uniform(0.5, 1.0)
        img += amp * np.sin(2.0 * np.pi * (xx * np.cos(theta) + yy * np.sin(theta)) / per + phase)
    lo, hi = img.min(), img.max()
    img = (img - lo) / max(hi - lo, 1e-12) * 255.0
    lo_side = max(1, size // 32)
    hi_side = max(lo_side + 1, size // 6)
    for _ in range(n_rects):
        w = int(rng.integers(lo_side, hi_side + 1))
        h = int(rng.integers(lo_side, hi_side + 1))
        x0 = int(rng.integers(0, max(1, size - w + 1)))
        y0 = int(rng.integers(0, max(1, size - h + 1)))
        img[y0:y0 + h, x0:x0 + w] = rng.uniform(0.0, 255.0)
    return img.astype(np.float32)


def add_gaussian(clean: np.ndarray, sigma: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng([seed, 0x6A55])
    return (clean.astype(np.float64) + rng.normal(0.0, sigma, clean.shape)).astype(np.float32)


def add_speckle(clean: np.ndarray, looks: float, seed: int) -> np.ndarray:
    """Multiplicative Gamma noise with shape ``looks`` and mean 1."""
    rng = np.random.default_rng([seed, 0x5BEC])
    g = rng.gamma(shape=looks, scale=1.0 / looks, size=clean.shape)
    return (clean.astype(np.float64) * g).astype(np.float32)


def psnr(ref: np.ndarray, img: np.ndarray, peak: float = 255.0) -> float:
    mse = float(np.mean((ref.astype(np.float64) - img.astype(np.float64)) ** 2))
    return float("inf") if mse == 0.0 else 10.0 * np.log10(peak * peak / mse)


def psnr_normalised(ref: np.ndarray, img: np.ndarray) -> float:
    """PSNR after the reference's min-max normalisation of the output to
    [0, 255] (denoiser.cpp:75, 95-96)."""
    img = img.astype(np.float64)
    lo, hi = img.min(), img.max()
    norm = (img - lo) / max(hi - lo, 1e-12) * 255.0
    return psnr(ref, norm)


@dataclass(frozen=True)
class Workload:
    """One synthetic denoising problem with the reference's parameters."""
    name: str
    size: int
    sigma: float
    patch: int
    stride: int
    atoms: int
    omp_iter: int
    ksvd_iter: int
    seed: int = 1234

    @property
    def n(self) -> int:
        return self.patch * self.patch

    @property
    def num_patches(self) -> int:
        m = (self.size - self.patch) // self.stride + 1
        return m * m

    def images(self):
        clean = clean_image(self.size, self.seed)
        return clean, add_gaussian(clean, self.sigma, self.seed)


# The three single-image workloads: 512^2 (sigma 20, 12x12 stride 3, 256
# atoms, L=5, 10 iterations), 2048^2 (sigma 25, same patches), 4096^2 (sigma
# 15, 16x16 stride 2, 512 atoms, L=8, 8 iterations).
WORKLOADS = {
    "img512_p12s3_k256": Workload("img512_p12s3_k256", 512, 20.0, 12, 3, 256, 5, 10),
    "img2048_p12s3_k256": Workload("img2048_p12s3_k256", 2048, 25.0, 12, 3, 256, 5, 10),
    "img4096_p16s2_k512": Workload("img4096_p16s2_k512", 4096, 15.0, 16, 2, 512, 8, 8),
    # profiling case: the 2048^2 shape at 1536^2 (259,081 patches, a 149 MB
    # patch matrix: larger than L2, a few hundred MB on the device)
    "img1536_p12s3_k256": Workload("img1536_p12s3_k256", 1536, 25.0, 12, 3, 256, 5, 10),
}


def many_workload(count: int = 64, seed: int = 2024, sides=(256, 512, 1024, 1536, 2048), patches=(8, 12, 22),
                  stride: int = 3, speckle_count: int = 16, atoms: int = 256, omp_iter: int = 5, ksvd_iter: int = 10):
    """The uneven batch: `count` seeded images with sides drawn uniformly from
    `sides`, patch sides from `patches` at `stride`; the first `speckle_count`
    (in a seeded order) get multiplicative Gamma noise of shape 4 (denoised in
    the log2 domain), the others Gaussian noise with sigma uniform in [10, 40].
    Returns a list of dicts: clean, noisy, side, patch, speckle, sigma2 (the
    noise variance handed to the denoiser; for speckle the variance of log2 of
    Gamma(4, 1/4) noise)."""
    rng = np.random.default_rng(seed)
    speck = set(rng.permutation(count)[:speckle_count].tolist())
    # variance of log2(g), g ~ Gamma(shape 4, mean 1): trigamma(4) / ln(2)^2
    trigamma4 = np.pi ** 2 / 6.0 - (1.0 + 1.0 / 4.0 + 1.0 / 9.0)
    var_log2 = trigamma4 / np.log(2.0) ** 2
    out = []
    for i in range(count):
        side = int(rng.choice(sides))
        patch = int(rng.choice(patches))
        img_seed = int(rng.integers(0, 2 ** 31 - 1))
        clean = clean_image(side, img_seed)
        if i in speck:
            clean = clean + 1.0  # strictly positive for the log domain
            noisy = add_speckle(clean, 4.0, img_seed)
            out.append(dict(clean=clean, noisy=noisy, side=side, patch=patch, stride=stride, speckle=True,
                            sigma2=float(var_log2), atoms=atoms, omp_iter=omp_iter, ksvd_iter=ksvd_iter))
        else:
            sigma = float(rng.uniform(10.0, 40.0))
            noisy = add_gaussian(clean, sigma, img_seed)
            out.append(dict(clean=clean, noisy=noisy, side=side, patch=patch, stride=stride, speckle=False,
                            sigma2=sigma * sigma, atoms=atoms, omp_iter=omp_iter, ksvd_iter=ksvd_iter))
    return out
