"""Accuracy of a K-SVD run against the FP64 oracle.

TEST INFRASTRUCTURE ONLY (the checker): used by tests/ and by bench.py's
quality report, which runs after every timed region.  The product library
never imports this module.

The FP64 reference is the oracle's K-SVD (oracle/ksvd_oracle.cpp, restating
cuda_svd_denoiser.cu:368-408 with CuBlasMatrixOmp::work,
cublas_matrix_omp.cu:107-402, and updateDictionary, cuda_svd_denoiser.cu:
285-362) started from the FP32 initial dictionary that the GPU path builds
(bit-exact with the oracle's FP32 initDictionary), so both sides start from
the same atoms.  What is compared:

* the first OMP call (the initial dictionary): the fraction of patches whose
  ordered support equals the FP64 one, and the largest coefficient error of
  the agreeing patches relative to the patch's largest FP64 coefficient;
* the first update sweep, run by both sides from the FP64 codes: the largest
  atom error ||d - d64|| / ||d64|| (up to sign) and the largest coefficient
  error relative to the patch's largest coefficient;
* the denoised image after the full run (T iterations, final OMP, rebuild):
  the PSNR against the clean image, beside the FP64 oracle's.
"""

from __future__ import annotations

import numpy as np


def support_agreement(idx: np.ndarray, ref_idx: np.ndarray) -> float:
    """Fraction of patches whose ordered support equals the reference's."""
    return float(np.mean(np.all(idx == ref_idx, axis=1)))


def coef_rel_err(idx, coef, ref_idx, ref_coef) -> float:
    """Largest |c - c_ref| / max|c_ref| over the patches with equal supports."""
    m = np.all(idx == ref_idx, axis=1)
    if not np.any(m):
        return float("inf")
    c, r = np.asarray(coef, np.float64)[m], np.asarray(ref_coef, np.float64)[m]
    scale = np.abs(r).max(axis=1, keepdims=True) + 1e-30
    return float((np.abs(c - r) / scale).max())


def atom_err(D: np.ndarray, ref_D: np.ndarray) -> float:
    """Largest ||d - d_ref|| / ||d_ref|| over the atoms, up to sign."""
    D = np.asarray(D, np.float64)
    R = np.asarray(ref_D, np.float64)
    nr = np.linalg.norm(R, axis=1) + 1e-300
    e = np.minimum(np.linalg.norm(D - R, axis=1), np.linalg.norm(D + R, axis=1)) / nr
    return float(e.max())


def fp64_reference(oracle, noisy, D0_f32, *, patch, stride, omp_iter, ksvd_iter, q1_cap, sigma2):
    """The FP64 oracle's K-SVD from the FP32 initial dictionary D0_f32.

    Returns a dict: Y (FP32 patches), idx0/coef0 (first OMP), D1/coef1 (first
    sweep from idx0/coef0), image (denoised after ksvd_iter iterations)."""
    Y = oracle.extract_patches(noisy, patch, patch, stride, stride)
    Y64 = Y.astype(np.float64)
    D = np.asarray(D0_f32, np.float64).copy()
    out = {"Y": Y}
    for it in range(ksvd_iter):
        idx, coef = oracle.omp(Y64, D, omp_iter, dtype=np.float64)
        if it == 0:
            out["idx0"], out["coef0"] = idx, coef
        D, coef = oracle.update_dictionary(Y64, D, idx, coef, q1_cap, dtype=np.float64)
        if it == 0:
            out["D1"], out["coef1"] = D.copy(), coef.copy()
    idx, coef = oracle.omp(Y64, D, omp_iter, dtype=np.float64)
    img, lam = oracle.build_image(np.asarray(noisy, np.float32), patch, patch, stride, stride, D, idx, coef,
                                  sigma2, False, dtype=np.float64)
    out["image"], out["lambda"] = img, lam
    if ksvd_iter == 0:
        out["idx0"], out["coef0"] = idx, coef
    return out
