"""ctypes bindings to the CPU oracle (oracle/ksvd_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
and by bench.py's CPU-baseline / reference arm.  The product library never
imports this module.

Array conventions follow the reference's column-major matrices
(newfla/CUDA-K-SVD-Denoising, src/lib/baseUtilityLib/baseUtilityLib.h:16-36):
patches are (N, n) row-major here, i.e. the reference's n x N column-major
matrix; the dictionary is (K, n), i.e. its n x K matrix; sparse codes are the
compact pair idx (N, L) int32 / coef (N, L).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB_PATH = _HERE / "libksvd_oracle.so"
_lib = None

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64
_int = ctypes.c_int


def build() -> Path:
    """Compile the oracle (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(_HERE)], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(_LIB_PATH))
        L.ko_set_threads.argtypes = [_int]
        L.ko_max_threads.restype = _int
        L.ko_num_patches.argtypes = [_int] * 6
        L.ko_num_patches.restype = _i64
        L.ko_extract_patches.argtypes = [_f32p] + [_int] * 6 + [_f32p]
        L.ko_extract_patches.restype = _int
        L.ko_init_dictionary_f32.argtypes = [_f32p, _i64, _int, _int, _int, _f32p]
        L.ko_init_dictionary_f64.argtypes = [_f64p, _i64, _int, _int, _int, _f64p]
        L.ko_omp_f32.argtypes = [_f32p, _i64, _int, _f32p, _int, _int, _i32p, _f32p]
        L.ko_omp_f64.argtypes = [_f64p, _i64, _int, _f64p, _int, _int, _i32p, _f64p]
        L.ko_update_f32.argtypes = [_f32p, _i64, _int, _f32p, _int, _int, _i32p, _f32p, _int]
        L.ko_update_f64.argtypes = [_f64p, _i64, _int, _f64p, _int, _int, _i32p, _f64p, _int]
        L.ko_build_image_f32.argtypes = ([_f32p] + [_int] * 6 + [_f32p, _int, _int, _i32p, _f32p,
                                          ctypes.c_double, _int, _f32p, ctypes.POINTER(ctypes.c_double)])
        L.ko_build_image_f64.argtypes = ([_f32p] + [_int] * 6 + [_f64p, _int, _int, _i32p, _f64p,
                                          ctypes.c_double, _int, _f32p, ctypes.POINTER(ctypes.c_double)])
        L.ko_sym_top_eig.argtypes = [_f64p, _int, _f64p]
        L.ko_sym_top_eig.restype = ctypes.c_double
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().ko_set_threads(int(n))


def max_threads() -> int:
    return int(lib().ko_max_threads())


def num_patches(W, H, pw, ph, sw, sh) -> int:
    return int(lib().ko_num_patches(W, H, pw, ph, sw, sh))


def extract_patches(img: np.ndarray, pw: int, ph: int, sw: int, sh: int) -> np.ndarray:
    """createPatches (cuda_svd_denoiser.cu:221-256). img is (H, W) row-major."""
    img = np.ascontiguousarray(img, dtype=np.float32)
    H, W = img.shape
    N = num_patches(W, H, pw, ph, sw, sh)
    if N < 0:
        raise ValueError("patch geometry does not fit the image")
    out = np.empty((N, pw * ph), np.float32)
    if lib().ko_extract_patches(img, W, H, pw, ph, sw, sh, out) != 0:
        raise ValueError("extract_patches failed")
    return out


def _dt(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def init_dictionary(patches: np.ndarray, K: int, int_norm: bool = True, dtype=np.float64) -> np.ndarray:
    """initDictionary (cuda_svd_denoiser.cu:261-280)."""
    P = np.ascontiguousarray(patches, dtype=dtype)
    N, n = P.shape
    D = np.empty((K, n), dtype)
    rc = getattr(lib(), "ko_init_dictionary_" + _dt(dtype))(P, N, n, K, int(bool(int_norm)), D)
    if rc == -1:
        raise ValueError("not enough patches for the initial dictionary")
    if rc == -2:
        raise FloatingPointError("zero-norm initial atom")
    return D


def omp(Y: np.ndarray, D: np.ndarray, L: int, dtype=np.float64):
    """CuBlasMatrixOmp::work (cublas_matrix_omp.cu:107-402) -> (idx, coef)."""
    Y = np.ascontiguousarray(Y, dtype=dtype)
    D = np.ascontiguousarray(D, dtype=dtype)
    N, n = Y.shape
    K = D.shape[0]
    idx = np.empty((N, L), np.int32)
    coef = np.empty((N, L), dtype)
    rc = getattr(lib(), "ko_omp_" + _dt(dtype))(Y, N, n, D, K, L, idx, coef)
    if rc != 0:
        raise ValueError("omp failed")
    return idx, coef


def update_dictionary(Y, D, idx, coef, q1_cap: bool, dtype=np.float64):
    """updateDictionary (cuda_svd_denoiser.cu:285-362) -> (D', coef')."""
    Y = np.ascontiguousarray(Y, dtype=dtype)
    D2 = np.array(D, dtype=dtype, copy=True, order="C")
    c2 = np.array(coef, dtype=dtype, copy=True, order="C")
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    N, n = Y.shape
    K = D2.shape[0]
    L = idx.shape[1]
    rc = getattr(lib(), "ko_update_" + _dt(dtype))(Y, N, n, D2, K, L, idx, c2, int(bool(q1_cap)))
    if rc != 0:
        raise ValueError("update failed")
    return D2, c2


def build_image(noisy: np.ndarray, pw, ph, sw, sh, D, idx, coef, sigma2: float, speckle: bool = False,
                dtype=np.float64):
    """createImage (cuda_svd_denoiser.cu:413-498) -> (image, lambda).

    ``noisy`` is the (log-domain for speckle) noisy image (H, W)."""
    noisy = np.ascontiguousarray(noisy, dtype=np.float32)
    H, W = noisy.shape
    D = np.ascontiguousarray(D, dtype=dtype)
    coef = np.ascontiguousarray(coef, dtype=dtype)
    idx = np.ascontiguousarray(idx, dtype=np.int32)
    out = np.empty((H, W), np.float32)
    lam = ctypes.c_double(0.0)
    rc = getattr(lib(), "ko_build_image_" + _dt(dtype))(noisy, W, H, pw, ph, sw, sh, D, D.shape[0],
                                                        idx.shape[1], idx, coef, float(sigma2),
                                                        int(bool(speckle)), out, ctypes.byref(lam))
    if rc != 0:
        raise ValueError("build_image failed")
    return out, lam.value


def sym_top_eig(A: np.ndarray):
    A = np.ascontiguousarray(A, dtype=np.float64)
    n = A.shape[0]
    u = np.empty(n, np.float64)
    lam = lib().ko_sym_top_eig(A, n, u)
    return lam, u


def my_log(img: np.ndarray) -> np.ndarray:
    """myLog (denoisingLib.h:124-133): log2, with 0 mapped to 0."""
    img = np.asarray(img, np.float32)
    out = np.zeros_like(img)
    nz = img != 0
    out[nz] = np.log2(img[nz])
    return out


def ksvd_denoise(noisy: np.ndarray, sigma2: float, *, pw=8, ph=8, sw=2, sh=2, atoms=256, ksvd_iter=10,
                 omp_iter=5, speckle=False, q1_cap=True, int_norm=True, dtype=np.float64):
    """internalDenoising without sub-images (cuda_svd_denoiser.cu:189-206) and
    kSvd (:368-408): T x (OMP + update), final OMP, createImage.

    Returns (image, info) where info holds the dictionary and codes."""
    y = my_log(noisy) if speckle else np.asarray(noisy, np.float32)
    Y = extract_patches(y, pw, ph, sw, sh)
    D = init_dictionary(Y, atoms, int_norm=int_norm, dtype=dtype)
    for _ in range(ksvd_iter):
        idx, coef = omp(Y, D, omp_iter, dtype=dtype)
        D, coef = update_dictionary(Y, D, idx, coef, q1_cap, dtype=dtype)
    idx, coef = omp(Y, D, omp_iter, dtype=dtype)
    out, lam = build_image(y, pw, ph, sw, sh, D, idx, coef, sigma2, speckle, dtype=dtype)
    return out, {"D": D, "idx": idx, "coef": coef, "lambda": lam}


if os.environ.get("KSVD_ORACLE_THREADS"):
    set_threads(int(os.environ["KSVD_ORACLE_THREADS"]))


def ksvd_denoise_tiled(noisy: np.ndarray, sigma2: float, sub_w: int, sub_h: int, **kw):
    """Sub-image mode (cuda_svd_denoiser.cu:130-188, 503-528): non-overlapping
    sub-images of sub_h (along x, the column index) by sub_w (along y, the
    row index) at a step of their own size, each denoised on its own with the
    same sigma2; pixels outside the complete sub-images are returned as the
    input.  Returns (image, mean lambda)."""
    H, W = noisy.shape
    out = np.array(noisy, dtype=np.float32, copy=True)
    lams = []
    for x0 in range(0, W - sub_h + 1, sub_h):
        for y0 in range(0, H - sub_w + 1, sub_w):
            tile = np.ascontiguousarray(noisy[y0:y0 + sub_w, x0:x0 + sub_h])
            r, info = ksvd_denoise(tile, sigma2, **kw)
            out[y0:y0 + sub_w, x0:x0 + sub_h] = r
            lams.append(info["lambda"])
    return out, float(np.mean(lams))


def compact_to_dense(idx: np.ndarray, coef: np.ndarray, K: int) -> np.ndarray:
    """Compact codes (N, L) -> dense (N, K); unused slots (idx < 0) skipped."""
    N, L = idx.shape
    out = np.zeros((N, K), dtype=np.float64)
    rows = np.repeat(np.arange(N), L)
    m = idx.reshape(-1) >= 0
    out[rows[m], idx.reshape(-1)[m]] = coef.reshape(-1)[m]
    return out
