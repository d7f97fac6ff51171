"""ctypes bindings to the ksvd_sm100 C ABI (include/ksvd_sm100.h).

Device buffers are torch CUDA tensors (torch provides device memory and
streams only); every computation runs in libksvd_sm100.so.  There is no CPU
fallback: if the library or a GPU is missing the calls raise.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libksvd_sm100.so"
HEADER = PKG_DIR.parent / "include" / "ksvd_sm100.h"

# ksvd_type
CUDA_K_GESVD, CUDA_K_GESVDJ, CUDA_K_GESVDA, CUDA_K_SM100A = 0, 1, 2, 3
# ksvd_status
OK, ERR_LOAD, ERR_DENOISE, ERR_SAVE = 0, -1, -2, -3
ERR_INVALID, ERR_CUDA, ERR_NO_MEMORY, ERR_TIMEOUT, ERR_NUMERIC, ERR_NO_DEVICE = -10, -11, -12, -13, -14, -15
ERR_TOO_LARGE = -16
# ksvd_precision
PREC_FP32, PREC_BF16_RESCORE, PREC_FP16_RESCORE, PREC_BF16_LEARNED = 0, 1, 2, 3
# learned proposal
PROPOSAL_HIDDEN, PROPOSAL_CANDIDATES, PROPOSAL_FALLBACK = 512, 16, 1.15
# compat flags
COMPAT_INT_NORM, COMPAT_Q1_CAP = 0x1, 0x2
COMPAT_REFERENCE = COMPAT_INT_NORM | COMPAT_Q1_CAP


class KsvdParams(ctypes.Structure):
    _fields_ = [
        ("patch_width_dim", ctypes.c_int),
        ("patch_height_dim", ctypes.c_int),
        ("sliding_width", ctypes.c_int),
        ("sliding_height", ctypes.c_int),
        ("atoms", ctypes.c_int),
        ("ksvd_iter", ctypes.c_int),
        ("omp_iter", ctypes.c_int),
        ("bw", ctypes.c_int),
        ("speckle", ctypes.c_int),
        ("type", ctypes.c_int),
        ("min_omp_iter_batch", ctypes.c_int),
        ("sub_image_width_dim", ctypes.c_int),
        ("sub_image_height_dim", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("compat", ctypes.c_uint),
        ("device", ctypes.c_int),
    ]


class KsvdStats(ctypes.Structure):
    _fields_ = [
        ("init_ms", ctypes.c_int64),
        ("working_ms", ctypes.c_int64),
        ("finalize_ms", ctypes.c_int64),
        ("num_patches", ctypes.c_int64),
        ("lambda_", ctypes.c_double),
        ("iter_ms", ctypes.c_double),
        ("final_omp_ms", ctypes.c_double),
        ("extract_ms", ctypes.c_double),
        ("build_ms", ctypes.c_double),
        ("power_iters", ctypes.c_int64),
        ("atoms_updated", ctypes.c_int64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class ProposalStats(ctypes.Structure):
    _fields_ = [
        ("pairs", ctypes.c_int64),
        ("steps", ctypes.c_int64),
        ("first_loss", ctypes.c_double),
        ("final_loss", ctypes.c_double),
        ("collect_ms", ctypes.c_double),
        ("train_ms", ctypes.c_double),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class TuneResult(ctypes.Structure):
    _fields_ = [
        ("update_slice", ctypes.c_int),
        ("candidates", ctypes.c_int),
        ("slice", ctypes.c_int * 8),
        ("update_ms", ctypes.c_double * 8),
    ]

    def as_dict(self) -> dict:
        k = self.candidates
        return {"update_slice": self.update_slice,
                "update_ms_by_slice": {int(self.slice[i]): float(self.update_ms[i]) for i in range(k)}}


class ImageJob(ctypes.Structure):
    _fields_ = [
        ("params", KsvdParams),
        ("img", ctypes.c_void_p),
        ("out", ctypes.c_void_p),
        ("width", ctypes.c_int),
        ("height", ctypes.c_int),
        ("sigma2", ctypes.c_float),
    ]


class ManyStats(ctypes.Structure):
    _fields_ = [
        ("num_patches", ctypes.c_int64),
        ("iter_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("graph", ctypes.c_int),
        ("streams", ctypes.c_int),
        ("plan_ms", ctypes.c_double),
        ("update_ctas", ctypes.c_int * 64),
        ("setup_ms", ctypes.c_double),
        ("tune_ms", ctypes.c_double),
        ("final_ms", ctypes.c_double),
        ("codes_ms", ctypes.c_double),
        ("sweep_ms", ctypes.c_double),
        ("lanes", ctypes.c_int),
        ("update_cta_begin", ctypes.c_int * 64),
    ]

    def as_dict(self, count: int) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("update_ctas", "update_cta_begin")}
        d["update_ctas"] = [int(self.update_ctas[i]) for i in range(count)]
        d["update_cta_begin"] = [int(self.update_cta_begin[i]) for i in range(count)]
        return d


class KsvdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"ksvd status {status}: {message}")
        self.status = status


_lib = None
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_int = ctypes.c_int


def build() -> Path:
    """Compile libksvd_sm100.so in-tree (make -C <package>)."""
    subprocess.run(["make", "-s", "-j8", "-C", str(PKG_DIR)], check=True)
    return LIB_PATH


def lib():
    """Load the library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with make -C {PKG_DIR}")
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.POINTER(KsvdParams)
        L.ksvd_abi_version.restype = _int
        L.ksvd_params_default.argtypes = [P]
        L.ksvd_type_from_string.argtypes = [ctypes.c_char_p, ctypes.POINTER(_int)]
        L.ksvd_type_from_string.restype = _int
        L.ksvd_type_name.argtypes = [_int]
        L.ksvd_type_name.restype = ctypes.c_char_p
        L.ksvd_status_string.argtypes = [_int]
        L.ksvd_status_string.restype = ctypes.c_char_p
        L.ksvd_num_patches.argtypes = [P, _int, _int]
        L.ksvd_num_patches.restype = _i64
        L.ksvd_create.argtypes = [P, ctypes.POINTER(_vp)]
        L.ksvd_create.restype = _int
        L.ksvd_destroy.argtypes = [_vp]
        L.ksvd_last_error.argtypes = [_vp]
        L.ksvd_last_error.restype = ctypes.c_char_p
        L.ksvd_set_stream.argtypes = [_vp, _vp]
        L.ksvd_set_stream.restype = _int
        L.ksvd_get_stream.argtypes = [_vp]
        L.ksvd_get_stream.restype = _vp
        L.ksvd_denoise.argtypes = [_vp, _vp, _int, _int, ctypes.c_float, _vp, ctypes.POINTER(KsvdStats)]
        L.ksvd_denoise.restype = _int
        L.ksvd_extract_patches.argtypes = [_vp, _vp, _int, _int, _vp]
        L.ksvd_extract_patches.restype = _int
        L.ksvd_init_dictionary.argtypes = [_vp, _vp, _i64, _vp]
        L.ksvd_init_dictionary.restype = _int
        L.ksvd_omp.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp]
        L.ksvd_omp.restype = _int
        L.ksvd_update_dictionary.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp]
        L.ksvd_update_dictionary.restype = _int
        L.ksvd_iterate.argtypes = [_vp, _vp, _i64, _vp, _vp, _vp, _int]
        L.ksvd_iterate.restype = _int
        L.ksvd_build_image.argtypes = [_vp, _vp, _int, _int, ctypes.c_float, _vp, _vp, _vp, _i64, _vp,
                                       ctypes.POINTER(ctypes.c_double)]
        L.ksvd_build_image.restype = _int
        L.ksvd_codes_to_dense.argtypes = [_vp, _vp, _vp, _i64, _vp]
        L.ksvd_codes_to_dense.restype = _int
        L.ksvd_profile_enable.argtypes = [_vp, _int]
        L.ksvd_profile_enable.restype = _int
        L.ksvd_profile_read.argtypes = [_vp, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(_i64)]
        L.ksvd_profile_read.restype = _int
        L.ksvd_profile_reset.argtypes = [_vp]
        L.ksvd_profile_reset.restype = _int
        L.ksvd_launch_count.argtypes = [_vp]
        L.ksvd_launch_count.restype = _i64
        L.ksvd_profile_phases.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), _int]
        L.ksvd_profile_phases.restype = _int
        L.ksvd_profile_counters.argtypes = [_vp, ctypes.POINTER(_i64), _int]
        L.ksvd_profile_counters.restype = _int
        L.ksvd_batch_count.argtypes = [ctypes.c_char_p]
        L.ksvd_batch_count.restype = _int
        L.ksvd_batch_entry.argtypes = [ctypes.c_char_p, _int, P, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                       ctypes.c_size_t, ctypes.POINTER(ctypes.c_double)]
        L.ksvd_batch_entry.restype = _int
        L.ksvd_run_batch.argtypes = [ctypes.c_char_p, _int]
        L.ksvd_run_batch.restype = _int
        L.ksvd_omp_noalloc.argtypes = [P, _vp, _i64, _vp, _vp, _vp, _vp]
        L.ksvd_omp_noalloc.restype = _int
        _u64 = ctypes.c_uint64
        PS = ctypes.POINTER(ProposalStats)
        L.ksvd_proposal_num_params.argtypes = [P]
        L.ksvd_proposal_num_params.restype = _i64
        L.ksvd_proposal_init.argtypes = [_vp, _u64]
        L.ksvd_proposal_init.restype = _int
        L.ksvd_proposal_set_params.argtypes = [_vp, _vp, _i64]
        L.ksvd_proposal_set_params.restype = _int
        L.ksvd_proposal_get_params.argtypes = [_vp, _vp, _i64]
        L.ksvd_proposal_get_params.restype = _int
        L.ksvd_proposal_loss_grad.argtypes = [_vp, _vp, _i64, _vp, ctypes.POINTER(ctypes.c_double), _vp]
        L.ksvd_proposal_loss_grad.restype = _int
        L.ksvd_proposal_train.argtypes = [_vp, _vp, _i64, _vp, _int, _int, _int, ctypes.c_float, _u64, PS]
        L.ksvd_proposal_train.restype = _int
        L.ksvd_proposal_fit.argtypes = [_vp, _vp, _i64, _vp, _int, _int, _u64, PS]
        L.ksvd_proposal_fit.restype = _int
        L.ksvd_proposal_candidates.argtypes = [_vp, _vp, _i64, _vp]
        L.ksvd_proposal_candidates.restype = _int
        L.ksvd_omp_restricted.argtypes = [_vp, _vp, _i64, _vp, _vp, _int, _vp, _vp, ctypes.POINTER(_i64)]
        L.ksvd_omp_restricted.restype = _int
        L.ksvd_set_noise_variance.argtypes = [_vp, ctypes.c_float]
        L.ksvd_set_noise_variance.restype = _int
        L.ksvd_proposal_fallbacks.argtypes = [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i64), ctypes.POINTER(_i64)]
        L.ksvd_proposal_fallbacks.restype = _int
        L.ksvd_autotune.argtypes = [_vp, _vp, _i64, _vp, ctypes.POINTER(TuneResult)]
        L.ksvd_autotune.restype = _int
        L.ksvd_set_update_slice.argtypes = [_vp, _int]
        L.ksvd_set_update_slice.restype = _int
        L.ksvd_denoise_many.argtypes = [ctypes.POINTER(ImageJob), _int, _int, _int, ctypes.POINTER(ManyStats)]
        L.ksvd_denoise_many.restype = _int
        L.ksvd_many_plan.argtypes = [ctypes.POINTER(ImageJob), _int, _int, ctypes.POINTER(_int), ctypes.POINTER(_int),
                                     ctypes.POINTER(_int), ctypes.POINTER(ctypes.c_double)]
        L.ksvd_many_plan.restype = _int
        _lib = L
    return _lib


def default_params() -> KsvdParams:
    p = KsvdParams()
    lib().ksvd_params_default(ctypes.byref(p))
    return p


def make_params(**kw) -> KsvdParams:
    p = default_params()
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, int(v))
    return p


def type_from_string(name: str):
    known = _int(0)
    t = lib().ksvd_type_from_string(name.encode(), ctypes.byref(known))
    return t, bool(known.value)


def num_patches(params: KsvdParams, width: int, height: int) -> int:
    return int(lib().ksvd_num_patches(ctypes.byref(params), width, height))


def _ptr(t) -> int:
    """Device pointer of a torch tensor (checked to be CUDA + contiguous)."""
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return t.data_ptr()


class Context:
    """Owns one ksvd_ctx.  Stage methods take torch CUDA tensors."""

    def __init__(self, params: KsvdParams | None = None, **kw):
        self.params = params if params is not None else make_params(**kw)
        h = _vp()
        st = lib().ksvd_create(ctypes.byref(self.params), ctypes.byref(h))
        if st != OK:
            raise KsvdError(st, lib().ksvd_status_string(st).decode())
        self.h = h

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            lib().ksvd_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != OK:
            raise KsvdError(st, lib().ksvd_last_error(self.h).decode())

    # -- properties -------------------------------------------------------
    @property
    def n(self) -> int:
        return self.params.patch_width_dim * self.params.patch_height_dim

    @property
    def K(self) -> int:
        return self.params.atoms

    @property
    def L(self) -> int:
        return self.params.omp_iter

    def set_stream(self, stream_handle: int | None):
        self._check(lib().ksvd_set_stream(self.h, stream_handle))

    # -- stages (device tensors) ------------------------------------------
    def extract_patches(self, img, out):
        H, W = img.shape
        self._check(lib().ksvd_extract_patches(self.h, _ptr(img), W, H, _ptr(out)))

    def init_dictionary(self, patches, dict_out):
        self._check(lib().ksvd_init_dictionary(self.h, _ptr(patches), patches.shape[0], _ptr(dict_out)))

    def omp(self, patches, dictionary, idx, coef):
        self._check(lib().ksvd_omp(self.h, _ptr(patches), patches.shape[0], _ptr(dictionary), _ptr(idx),
                                   _ptr(coef)))

    def update_dictionary(self, patches, dictionary, idx, coef):
        self._check(lib().ksvd_update_dictionary(self.h, _ptr(patches), patches.shape[0], _ptr(dictionary),
                                                 _ptr(idx), _ptr(coef)))

    def iterate(self, patches, dictionary, idx, coef, iters: int):
        self._check(lib().ksvd_iterate(self.h, _ptr(patches), patches.shape[0], _ptr(dictionary), _ptr(idx),
                                       _ptr(coef), int(iters)))

    def build_image(self, noisy, sigma2, dictionary, idx, coef, out) -> float:
        H, W = noisy.shape
        lam = ctypes.c_double(0.0)
        self._check(lib().ksvd_build_image(self.h, _ptr(noisy), W, H, float(sigma2), _ptr(dictionary), _ptr(idx),
                                           _ptr(coef), idx.shape[0], _ptr(out), ctypes.byref(lam)))
        return lam.value

    def codes_to_dense(self, idx, coef, dense):
        self._check(lib().ksvd_codes_to_dense(self.h, _ptr(idx), _ptr(coef), idx.shape[0], _ptr(dense)))

    # -- whole denoise (host buffers) -------------------------------------
    def denoise(self, img: np.ndarray, sigma2: float, out: np.ndarray | None = None):
        img = np.ascontiguousarray(img, dtype=np.float32)
        H, W = img.shape
        if out is None:
            out = np.empty_like(img)
        st = KsvdStats()
        self._check(lib().ksvd_denoise(self.h, img.ctypes.data, W, H, float(sigma2), out.ctypes.data,
                                       ctypes.byref(st)))
        return out, st.as_dict()

    def denoise_ptr(self, img_ptr: int, W: int, H: int, sigma2: float, out_ptr: int) -> KsvdStats:
        """Host-pointer form (e.g. pinned torch tensors)."""
        st = KsvdStats()
        self._check(lib().ksvd_denoise(self.h, img_ptr, W, H, float(sigma2), out_ptr, ctypes.byref(st)))
        return st

    # -- profiling --------------------------------------------------------
    def profile(self, level: int = 1):
        """0 off, 1 per-family event timing, 2 + in-kernel phase timers."""
        self._check(lib().ksvd_profile_enable(self.h, int(level)))

    def profile_reset(self):
        self._check(lib().ksvd_profile_reset(self.h))

    def profile_read(self, family: str):
        ms = ctypes.c_double(0.0)
        n = _i64(0)
        self._check(lib().ksvd_profile_read(self.h, family.encode(), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def profile_phases(self) -> list:
        arr = (ctypes.c_double * 16)()
        self._check(lib().ksvd_profile_phases(self.h, arr, 16))
        return list(arr)

    def profile_counters(self) -> dict:
        arr = (_i64 * 4)()
        self._check(lib().ksvd_profile_counters(self.h, arr, 4))
        return {"power_iters": arr[0], "atoms_updated": arr[1], "omp_window_overflows": arr[2],
                "omp_exact_rescores": arr[3]}

    def launch_count(self) -> int:
        return int(lib().ksvd_launch_count(self.h))

    # -- autotuning --------------------------------------------------------
    def autotune(self, patches, dictionary) -> dict:
        r = TuneResult()
        self._check(lib().ksvd_autotune(self.h, _ptr(patches), patches.shape[0], _ptr(dictionary),
                                        ctypes.byref(r)))
        return r.as_dict()

    def set_update_slice(self, slice_: int):
        self._check(lib().ksvd_set_update_slice(self.h, int(slice_)))

    # -- learned support proposal -----------------------------------------
    def proposal_num_params(self) -> int:
        return int(lib().ksvd_proposal_num_params(ctypes.byref(self.params)))

    def proposal_init(self, seed: int = 0):
        self._check(lib().ksvd_proposal_init(self.h, int(seed)))

    def proposal_set_params(self, params: np.ndarray):
        params = np.ascontiguousarray(params, dtype=np.float32)
        self._check(lib().ksvd_proposal_set_params(self.h, params.ctypes.data, params.size))

    def proposal_get_params(self) -> np.ndarray:
        out = np.empty(self.proposal_num_params(), np.float32)
        self._check(lib().ksvd_proposal_get_params(self.h, out.ctypes.data, out.size))
        return out

    def proposal_loss_grad(self, patches, supports, grad) -> float:
        loss = ctypes.c_double(0.0)
        self._check(lib().ksvd_proposal_loss_grad(self.h, _ptr(patches), patches.shape[0], _ptr(supports),
                                                  ctypes.byref(loss), _ptr(grad)))
        return loss.value

    def proposal_train(self, patches, supports, T: int, epochs: int, batch: int = 4096, lr: float = 1e-3,
                       seed: int = 0) -> dict:
        st = ProposalStats()
        self._check(lib().ksvd_proposal_train(self.h, _ptr(patches), patches.shape[0], _ptr(supports), int(T),
                                              int(epochs), int(batch), float(lr), int(seed), ctypes.byref(st)))
        return st.as_dict()

    def proposal_fit(self, patches, dictionary, iters: int, epochs: int = 2, seed: int = 0) -> dict:
        st = ProposalStats()
        self._check(lib().ksvd_proposal_fit(self.h, _ptr(patches), patches.shape[0], _ptr(dictionary), int(iters),
                                            int(epochs), int(seed), ctypes.byref(st)))
        return st.as_dict()

    def proposal_candidates(self, patches, cand):
        self._check(lib().ksvd_proposal_candidates(self.h, _ptr(patches), patches.shape[0], _ptr(cand)))

    def omp_restricted(self, patches, dictionary, cand, idx, coef) -> int:
        above = _i64(0)
        self._check(lib().ksvd_omp_restricted(self.h, _ptr(patches), patches.shape[0], _ptr(dictionary), _ptr(cand),
                                              cand.shape[1], _ptr(idx), _ptr(coef), ctypes.byref(above)))
        return above.value

    def set_noise_variance(self, sigma2: float):
        self._check(lib().ksvd_set_noise_variance(self.h, float(sigma2)))

    def proposal_fallbacks(self) -> dict:
        a, b, c = _i64(0), _i64(0), _i64(0)
        self._check(lib().ksvd_proposal_fallbacks(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return {"last": a.value, "total": b.value, "patches": c.value}


def denoise_many(jobs, device: int = 0, tune: bool = True, outs=None):
    """ksvd_denoise_many over [(params, image (H, W) float32, sigma2), ...].
    Returns (list of denoised images, stats dict)."""
    arr = (ImageJob * len(jobs))()
    keep = []
    out_list = []
    for i, (params, img, sigma2) in enumerate(jobs):
        img = np.ascontiguousarray(img, dtype=np.float32)
        out = outs[i] if outs is not None else np.empty_like(img)
        keep.append(img)
        out_list.append(out)
        arr[i].params = params
        arr[i].img = img.ctypes.data
        arr[i].out = out.ctypes.data
        arr[i].height, arr[i].width = img.shape
        arr[i].sigma2 = float(sigma2)
    st = ManyStats()
    rc = lib().ksvd_denoise_many(arr, len(jobs), int(device), int(bool(tune)), ctypes.byref(st))
    if rc != OK:
        raise KsvdError(rc, lib().ksvd_status_string(rc).decode())
    return out_list, st.as_dict(len(jobs))


def many_plan(shapes, num_sms: int = 148):
    """ksvd_many_plan over [(params, width, height), ...] (host only): the
    shared sweep's lane plan as (cta_begin, ctas, order, modelled ms)."""
    m = len(shapes)
    arr = (ImageJob * m)()
    for i, (params, width, height) in enumerate(shapes):
        arr[i].params = params
        arr[i].width, arr[i].height = int(width), int(height)
    b, c, o = (_int * m)(), (_int * m)(), (_int * m)()
    ms = ctypes.c_double(0.0)
    rc = lib().ksvd_many_plan(arr, m, int(num_sms), b, c, o, ctypes.byref(ms))
    if rc != OK:
        raise KsvdError(rc, lib().ksvd_status_string(rc).decode())
    return list(b), list(c), list(o), ms.value


def omp_noalloc(params: KsvdParams, patches, dictionary, idx, coef, stream_handle: int | None = None) -> int:
    """ksvd_omp_noalloc: OMP without a context or any device allocation
    (torch CUDA tensors on the current device).  Returns the status."""
    return int(lib().ksvd_omp_noalloc(ctypes.byref(params), _ptr(patches), patches.shape[0], _ptr(dictionary),
                                      _ptr(idx), _ptr(coef), stream_handle))


def batch_config(path: str) -> list[dict]:
    """Entries of a config.json as the library reads them (BatchDenoiser::factory)."""
    n = lib().ksvd_batch_count(str(path).encode())
    if n < 0:
        raise KsvdError(ERR_INVALID, f"cannot read {path}")
    out = []
    for i in range(n):
        p = KsvdParams()
        bufs = [ctypes.create_string_buffer(4096) for _ in range(3)]
        nv = ctypes.c_double(0.0)
        st = lib().ksvd_batch_entry(str(path).encode(), i, ctypes.byref(p), bufs[0], bufs[1], bufs[2], 4096,
                                    ctypes.byref(nv))
        if st != OK:
            raise KsvdError(st, f"entry {i} of {path}")
        d = {k: getattr(p, k) for k, _ in p._fields_}
        d.update(input=bufs[0].value.decode(), output=bufs[1].value.decode(), ref=bufs[2].value.decode(),
                 noise_variance=nv.value)
        out.append(d)
    return out


def run_batch(path: str, verbose: bool = False) -> int:
    return int(lib().ksvd_run_batch(str(path).encode(), int(verbose)))


def declared_symbols() -> list[str]:
    """Function names declared in include/ksvd_sm100.h."""
    import re
    txt = HEADER.read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(ksvd_[a-z0-9_]+)\s*\(", txt)))
