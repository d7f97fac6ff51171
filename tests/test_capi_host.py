"""Host-side checks of the C ABI: the library loads, exports every declared
symbol, and its host-only entry points behave (no GPU work)."""

import ctypes

import numpy as np

import pytest


def test_exports_every_declared_symbol(built_lib, ksvd):
    names = ksvd.declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(built_lib, n)]
    assert not missing, missing


def test_abi_version(built_lib):
    assert built_lib.ksvd_abi_version() == 1


def test_params_default_match_reference(ksvd, built_lib):
    # denoisingLib.h:44-56
    p = ksvd.default_params()
    assert (p.patch_width_dim, p.patch_height_dim) == (8, 8)
    assert (p.sliding_width, p.sliding_height) == (2, 2)
    assert (p.atoms, p.ksvd_iter, p.omp_iter) == (256, 10, 5)
    assert (p.sub_image_width_dim, p.sub_image_height_dim) == (0, 0)
    assert p.bw == 1 and p.speckle == 0 and p.min_omp_iter_batch == 0
    assert p.type == ksvd.CUDA_K_SM100A
    assert p.compat == ksvd.COMPAT_REFERENCE


def test_type_map(ksvd, built_lib):
    # DenoiserTypeMap (denoisingLib.h:23-31); unknown names map to 0 like
    # std::map::operator[]
    assert ksvd.type_from_string("CUDA_K_GESVD") == (0, True)
    assert ksvd.type_from_string("CUDA_K_GESVDJ") == (1, True)
    assert ksvd.type_from_string("CUDA_K_GESVDA") == (2, True)
    assert ksvd.type_from_string("CUDA_K_SM100A") == (3, True)
    assert ksvd.type_from_string("nonsense") == (0, False)
    assert built_lib.ksvd_type_name(1) == b"CUDA_K_GESVDJ"


def test_num_patches(ksvd, built_lib):
    p = ksvd.make_params(patch_width_dim=12, patch_height_dim=12, sliding_width=3, sliding_height=3)
    assert ksvd.num_patches(p, 512, 512) == 167 * 167
    assert ksvd.num_patches(p, 2048, 2048) == 679 * 679
    assert ksvd.num_patches(p, 11, 512) == -1


def test_status_strings(built_lib):
    assert built_lib.ksvd_status_string(0) == b"ok"
    assert built_lib.ksvd_status_string(-1) == b"image loading failed"
    assert built_lib.ksvd_status_string(-2) == b"denoising failed"
    assert built_lib.ksvd_status_string(-3) == b"image saving failed"


def test_create_rejects_bad_params(ksvd, built_lib):
    for kw in (dict(atoms=0), dict(omp_iter=0), dict(omp_iter=33), dict(sliding_width=0), dict(type=7)):
        p = ksvd.make_params(**kw)
        h = ctypes.c_void_p()
        assert built_lib.ksvd_create(ctypes.byref(p), ctypes.byref(h)) == ksvd.ERR_INVALID


def test_create_without_gpu_reports_no_device(ksvd, built_lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    p = ksvd.default_params()
    h = ctypes.c_void_p()
    assert built_lib.ksvd_create(ctypes.byref(p), ctypes.byref(h)) == ksvd.ERR_NO_DEVICE
    with pytest.raises(ksvd.KsvdError):
        ksvd.Context()


def test_null_context_is_rejected(built_lib, ksvd):
    assert built_lib.ksvd_omp(None, None, 0, None, None, None) == ksvd.ERR_INVALID
    assert built_lib.ksvd_last_error(None) == b"null context"


def test_noalloc_rejects_patch_areas_that_do_not_fit_an_int(ksvd, built_lib):
    """4 x (2^30 + 36) would wrap to 144 as a 32-bit product: rejected before
    any device work (the pointers are never touched)."""
    fake = ctypes.c_void_p(16)
    for pw, ph in ((4, 2 ** 30 + 36), (2 ** 16, 2 ** 16), (0, 8), (8, -1)):
        p = ksvd.make_params(patch_width_dim=pw, patch_height_dim=ph)
        st = built_lib.ksvd_omp_noalloc(ctypes.byref(p), fake, ctypes.c_int64(1000), fake, fake, fake, None)
        assert st == ksvd.ERR_INVALID, (pw, ph, st)


def _check_plan(b, c, o, count, sms):
    # every image once in the order; each image's range inside the grid;
    # images sharing a range share it exactly (a lane), and lanes are
    # disjoint and tile the grid
    assert sorted(o) == list(range(count))
    lanes = {}
    for i in range(count):
        assert c[i] >= 1 and 0 <= b[i] and b[i] + c[i] <= sms
        lanes.setdefault(b[i], set()).add(c[i])
    assert all(len(w) == 1 for w in lanes.values())
    spans = sorted((beg, beg + next(iter(w))) for beg, w in lanes.items())
    assert spans[0][0] == 0 and spans[-1][1] == sms
    assert all(spans[k][1] == spans[k + 1][0] for k in range(len(spans) - 1))
    # the images of a lane are consecutive in the sweep order
    seen = []
    for i in o:
        if not seen or seen[-1] != b[i]:
            assert b[i] not in seen
            seen.append(b[i])


def test_many_plan_lanes_tile_the_grid(ksvd, built_lib, synth):
    """ksvd_many_plan (the shared sweep's lane plan, host only) on the uneven
    64-image workload and on small cases: a valid plan, the small images not
    given a wide lane of their own, one image alone on every SM."""
    jobs = synth.many_workload(count=64)
    shapes = [(ksvd.make_params(patch_width_dim=j["patch"], patch_height_dim=j["patch"], sliding_width=j["stride"],
                                sliding_height=j["stride"], atoms=256, omp_iter=5), j["side"], j["side"]) for j in jobs]
    b, c, o, ms = ksvd.many_plan(shapes, 148)
    _check_plan(b, c, o, 64, 148)
    assert ms > 0 and len(set(b)) > 1
    b1, c1, o1, _ = ksvd.many_plan(shapes[:1], 148)
    assert (b1, c1, o1) == ([0], [148], [0])
    small = [(ksvd.make_params(patch_width_dim=8, patch_height_dim=8, sliding_width=3, sliding_height=3, atoms=64,
                               omp_iter=4), 96, 96)] * 5
    b5, c5, o5, _ = ksvd.many_plan(small, 20)
    _check_plan(b5, c5, o5, 5, 20)
    # subsets of every size: every lane gets an image (an empty lane hands
    # its CTAs to a neighbour), so the lanes always tile the grid
    rng = np.random.default_rng(7)
    for m in (2, 3, 5, 9, 17, 33):
        sub = [shapes[i] for i in rng.choice(64, size=m, replace=False)]
        bs, cs, os_, ms_s = ksvd.many_plan(sub, 148)
        _check_plan(bs, cs, os_, m, 148)
        assert ms_s > 0
    with pytest.raises(ksvd.KsvdError):
        ksvd.many_plan(shapes[:1], 0)
