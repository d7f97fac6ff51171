"""CUDA path against the CPU oracle, stage by stage and end to end, through
the C ABI.  Tolerances (stated per test) follow the targets: bit-exact for the
patch gather and the dictionary initialisation; OMP support agreement >= 99.9%
with coefficients within 1e-4 relative; atoms within 1e-4 (up to sign, the
sign convention is fixed); PSNR within 0.05 dB of the FP64 oracle."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mkctx(ksvd, **kw):
    return ksvd.Context(ksvd.make_params(**kw))


@pytest.fixture(scope="module")
def case(synth, oracle):
    clean = synth.clean_image(128, 21)
    noisy = synth.add_gaussian(clean, 20.0, 21)
    return clean, noisy


@pytest.fixture(scope="module")
def geo():
    return dict(patch_width_dim=8, patch_height_dim=8, sliding_width=2, sliding_height=2, atoms=64, omp_iter=5)


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_patches(torch, ksvd, img, **kw):
    c = mkctx(ksvd, **kw)
    H, W = img.shape
    N = ksvd.num_patches(c.params, W, H)
    out = torch.empty((N, c.n), dtype=torch.float32, device="cuda")
    c.extract_patches(dev(torch, img), out)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("pw,ph,sw,sh,size", [(8, 8, 2, 2, 128), (12, 12, 3, 3, 100), (16, 16, 2, 2, 66),
                                              (5, 7, 3, 2, 41), (12, 12, 3, 3, 512)])
def test_extract_patches_bitexact(torch_cuda, ksvd, synth, oracle, pw, ph, sw, sh, size):
    img = synth.add_gaussian(synth.clean_image(size, size), 25.0, 1)
    got = gpu_patches(torch_cuda, ksvd, img, patch_width_dim=pw, patch_height_dim=ph, sliding_width=sw,
                      sliding_height=sh, atoms=4).cpu().numpy()
    ref = oracle.extract_patches(img, pw, ph, sw, sh)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("compat", [0, 1, 3])
def test_init_dictionary_bitexact(torch_cuda, ksvd, oracle, case, geo, compat):
    _, noisy = case
    c = mkctx(ksvd, compat=compat, **geo)
    Y = oracle.extract_patches(noisy, 8, 8, 2, 2)
    D = torch_cuda.empty((c.K, c.n), dtype=torch_cuda.float32, device="cuda")
    c.init_dictionary(dev(torch_cuda, Y), D)
    ref = oracle.init_dictionary(Y, c.K, int_norm=bool(compat & 1), dtype=np.float32)
    np.testing.assert_array_equal(D.cpu().numpy(), ref)


def run_omp(torch, ksvd, Y, D, **kw):
    c = mkctx(ksvd, **kw)
    N = Y.shape[0]
    idx = torch.empty((N, c.L), dtype=torch.int32, device="cuda")
    coef = torch.empty((N, c.L), dtype=torch.float32, device="cuda")
    c.omp(dev(torch, Y), dev(torch, D), idx, coef)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), coef.cpu().numpy()


def support_agreement(i1, i2):
    return float(np.mean(np.all(i1 == i2, axis=1)))


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("K,L", [(64, 5), (32, 3), (256, 5), (100, 8)])
def test_omp_vs_fp64_oracle(torch_cuda, ksvd, oracle, case, K, L, precision):
    _, noisy = case
    Y = oracle.extract_patches(noisy, 8, 8, 2, 2)
    D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
    idx, coef = run_omp(torch_cuda, ksvd, Y, D, patch_width_dim=8, patch_height_dim=8, sliding_width=2,
                        sliding_height=2, atoms=K, omp_iter=L, precision=precision)
    ri, rc = oracle.omp(Y.astype(np.float64), D.astype(np.float64), L)
    agree = support_agreement(idx, ri)
    assert agree >= 0.999, agree
    m = np.all(idx == ri, axis=1)
    rel = np.abs(coef[m] - rc[m]) / (np.abs(rc[m]).max(axis=1, keepdims=True) + 1e-30)
    assert rel.max() < 1e-4, rel.max()


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_omp_img512_patches(torch_cuda, ksvd, oracle, synth, precision):
    """12x12 patches of the 512^2 workload image (27,889 patches, 144-dim),
    256 atoms, L = 5: support agreement with the FP64 oracle >= 99.9%."""
    w = synth.WORKLOADS["img512_p12s3_k256"]
    _, noisy = w.images()
    Y = oracle.extract_patches(noisy, 12, 12, 3, 3)
    D = oracle.init_dictionary(Y, 256, int_norm=True, dtype=np.float32)
    idx, coef = run_omp(torch_cuda, ksvd, Y, D, patch_width_dim=12, patch_height_dim=12, sliding_width=3,
                        sliding_height=3, atoms=256, omp_iter=5, precision=precision)
    ri, rc = oracle.omp(Y.astype(np.float64), D.astype(np.float64), 5)
    agree = support_agreement(idx, ri)
    assert agree >= 0.999, agree
    m = np.all(idx == ri, axis=1)
    rel = np.abs(coef[m] - rc[m]) / (np.abs(rc[m]).max(axis=1, keepdims=True) + 1e-30)
    assert rel.max() < 1e-4, rel.max()


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_omp_edge_cases(torch_cuda, ksvd, oracle, precision):
    # zero patches, exactly representable patches, fewer patches than a tile
    r = np.random.default_rng(5)
    D = r.normal(size=(40, 64)).astype(np.float32)
    D /= np.linalg.norm(D, axis=1, keepdims=True)
    Y = np.zeros((37, 64), np.float32)
    Y[1] = 3.0 * D[7]
    Y[2] = 2.0 * D[3] - 1.0 * D[11]
    Y[3:] = r.normal(scale=50.0, size=(34, 64))
    idx, coef = run_omp(torch_cuda, ksvd, Y, D, patch_width_dim=8, patch_height_dim=8, atoms=40, omp_iter=5,
                        precision=precision)
    ri, rc = oracle.omp(Y.astype(np.float64), D.astype(np.float64), 5)
    assert list(idx[0]) == [0, -1, -1, -1, -1] and coef[0, 0] == 0.0
    assert idx[1, 0] == 7 and abs(coef[1, 0] - 3.0) < 1e-5
    assert set(idx[2][:2]) == {3, 11}
    np.testing.assert_array_equal(idx[3:], ri[3:])
    np.testing.assert_allclose(coef[3:], rc[3:], rtol=1e-4, atol=1e-3)


def run_update(torch, ksvd, Y, D, idx, coef, **kw):
    c = mkctx(ksvd, **kw)
    Dd = dev(torch, D.astype(np.float32))
    cd = dev(torch, coef.astype(np.float32))
    c.update_dictionary(dev(torch, Y), Dd, dev(torch, idx), cd)
    torch.cuda.synchronize()
    return Dd.cpu().numpy(), cd.cpu().numpy()


@pytest.mark.parametrize("q1", [False, True])
def test_update_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, q1):
    clean = synth.clean_image(160, 8)
    noisy = synth.add_gaussian(clean, 20.0, 8)
    Y = oracle.extract_patches(noisy, 8, 8, 1, 1)  # 153^2 = 23409 patches: atoms with > 1024 users
    K, L = 64, 4
    D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, L, dtype=np.float32)
    assert np.bincount(idx[idx >= 0], minlength=K).max() > 1024
    kw = dict(patch_width_dim=8, patch_height_dim=8, sliding_width=1, sliding_height=1, atoms=K, omp_iter=L,
              compat=(3 if q1 else 1))
    Dg, cg = run_update(torch_cuda, ksvd, Y, D, idx, coef, **kw)
    Dr, cr = oracle.update_dictionary(Y.astype(np.float64), D.astype(np.float64), idx, coef.astype(np.float64),
                                      q1_cap=q1)
    err = np.abs(Dg - Dr).max()
    assert err < 1e-4, err
    np.testing.assert_allclose(np.linalg.norm(Dg, axis=1), 1.0, atol=1e-5)
    scale = np.abs(cr).max()
    assert np.abs(cg - cr).max() < 1e-4 * scale
    if q1:
        assert np.count_nonzero(cr == 0.0) > 0 and np.all(cg[cr == 0.0] == 0.0)


def test_update_keeps_unused_atoms(torch_cuda, ksvd, oracle, case):
    _, noisy = case
    Y = oracle.extract_patches(noisy, 8, 8, 2, 2)
    D = oracle.init_dictionary(Y, 64, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, 5, dtype=np.float32)
    used = np.zeros(64, bool)
    used[idx[(idx >= 0) & (coef != 0)]] = True
    idx2 = idx.copy()
    idx2[np.isin(idx2, [5, 9])] = -1  # atoms 5 and 9 lose every user
    Dg, _ = run_update(torch_cuda, ksvd, Y, D, idx2, coef, patch_width_dim=8, patch_height_dim=8,
                       sliding_width=2, sliding_height=2, atoms=64, omp_iter=5)
    np.testing.assert_array_equal(Dg[[5, 9]], D[[5, 9]])


def test_build_image_vs_oracle(torch_cuda, ksvd, oracle, case, geo):
    _, noisy = case
    Y = oracle.extract_patches(noisy, 8, 8, 2, 2)
    D = oracle.init_dictionary(Y, 64, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, 5, dtype=np.float32)
    c = mkctx(ksvd, **geo)
    out = torch_cuda.empty(noisy.shape, dtype=torch_cuda.float32, device="cuda")
    lam = c.build_image(dev(torch_cuda, noisy), 400.0, dev(torch_cuda, D), dev(torch_cuda, idx),
                        dev(torch_cuda, coef), out)
    ref, rlam = oracle.build_image(noisy, 8, 8, 2, 2, D, idx, coef, 400.0, dtype=np.float32)
    assert lam == pytest.approx(rlam, rel=1e-5)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-3)


def test_build_image_uncovered_border(torch_cuda, ksvd, oracle, synth):
    # 50 - 12 is not a multiple of 3: the last columns/rows are uncovered
    img = synth.add_gaussian(synth.clean_image(50, 2), 20.0, 2)
    Y = oracle.extract_patches(img, 12, 12, 3, 3)
    D = oracle.init_dictionary(Y, 16, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, 3, dtype=np.float32)
    c = mkctx(ksvd, patch_width_dim=12, patch_height_dim=12, sliding_width=3, sliding_height=3, atoms=16,
              omp_iter=3)
    out = torch_cuda.empty(img.shape, dtype=torch_cuda.float32, device="cuda")
    c.build_image(dev(torch_cuda, img), 400.0, dev(torch_cuda, D), dev(torch_cuda, idx), dev(torch_cuda, coef), out)
    o = out.cpu().numpy()
    assert np.all(np.isfinite(o))
    np.testing.assert_array_equal(o[:, 48:], img[:, 48:])
    ref, _ = oracle.build_image(img, 12, 12, 3, 3, D, idx, coef, 400.0, dtype=np.float32)
    np.testing.assert_allclose(o, ref, rtol=1e-5, atol=1e-3)


def test_codes_to_dense(torch_cuda, ksvd, oracle, case, geo):
    _, noisy = case
    Y = oracle.extract_patches(noisy, 8, 8, 2, 2)
    D = oracle.init_dictionary(Y, 64, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, 5, dtype=np.float32)
    c = mkctx(ksvd, **geo)
    N = Y.shape[0]
    dense = torch_cuda.empty((N, 64), dtype=torch_cuda.float32, device="cuda")
    c.codes_to_dense(dev(torch_cuda, idx), dev(torch_cuda, coef), dense)
    ref = np.zeros((N, 64), np.float32)
    for s in range(5):
        m = idx[:, s] >= 0
        ref[np.nonzero(m)[0], idx[m, s]] = coef[m, s]
    np.testing.assert_array_equal(dense.cpu().numpy(), ref)


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("compat,q1", [(1, False), (3, True)])
def test_denoise_psnr_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, compat, q1, precision):
    clean = synth.clean_image(128, 31)
    noisy = synth.add_gaussian(clean, 20.0, 31)
    kw = dict(patch_width_dim=8, patch_height_dim=8, sliding_width=2, sliding_height=2, atoms=64, omp_iter=5,
              ksvd_iter=4, compat=compat, precision=precision)
    with mkctx(ksvd, **kw) as c:
        out, st = c.denoise(noisy, 400.0)
    ref, info = oracle.ksvd_denoise(noisy, 400.0, pw=8, ph=8, sw=2, sh=2, atoms=64, ksvd_iter=4, omp_iter=5,
                                    q1_cap=q1, int_norm=True)
    pg, pr = synth.psnr(clean, out), synth.psnr(clean, ref)
    assert abs(pg - pr) <= 0.05, (pg, pr)
    assert pg > synth.psnr(clean, noisy) + 2.0
    assert st["num_patches"] == 61 * 61
    assert st["lambda_"] == pytest.approx(info["lambda"], rel=1e-2)


def test_denoise_speckle(torch_cuda, ksvd, oracle, synth):
    clean = synth.clean_image(96, 4) + 1.0
    noisy = synth.add_speckle(clean, 4.0, 4)
    kw = dict(patch_width_dim=8, patch_height_dim=8, sliding_width=2, sliding_height=2, atoms=32, omp_iter=4,
              ksvd_iter=2, speckle=1)
    with mkctx(ksvd, **kw) as c:
        out, _ = c.denoise(noisy, 0.3)
    ref, _ = oracle.ksvd_denoise(noisy, 0.3, pw=8, ph=8, sw=2, sh=2, atoms=32, ksvd_iter=2, omp_iter=4,
                                 speckle=True)
    assert np.all(np.isfinite(out))
    assert abs(synth.psnr(clean, out) - synth.psnr(clean, ref)) <= 0.05


def test_denoise_errors(torch_cuda, ksvd, synth):
    img = synth.clean_image(32, 1)
    with mkctx(ksvd, patch_width_dim=40, patch_height_dim=40, atoms=4) as c:
        with pytest.raises(ksvd.KsvdError) as e:
            c.denoise(img, 100.0)
        assert e.value.status == ksvd.ERR_INVALID
    with mkctx(ksvd, atoms=4000) as c:  # fewer patches than N/2 + K
        with pytest.raises(ksvd.KsvdError) as e:
            c.denoise(img, 100.0)
        assert e.value.status == ksvd.ERR_INVALID
    with mkctx(ksvd, atoms=16) as c:
        with pytest.raises(ksvd.KsvdError):
            c.denoise(img, 0.0)
        # the context stays usable after an error
        out, _ = c.denoise(img + 1.0, 100.0)
        assert np.all(np.isfinite(out))


def test_zero_image_reports_zero_atom(torch_cuda, ksvd):
    img = np.zeros((32, 32), np.float32)
    with mkctx(ksvd, atoms=16, ksvd_iter=1) as c:
        with pytest.raises(ksvd.KsvdError) as e:
            c.denoise(img, 100.0)
        assert e.value.status == ksvd.ERR_NUMERIC
        out, _ = c.denoise(np.ones((32, 32), np.float32) * 7.0, 100.0)
        np.testing.assert_allclose(out, 7.0, rtol=1e-5)


@pytest.mark.slow
@pytest.mark.parametrize("precision", [0, 1, 2])
def test_denoise_img512_workload_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, precision):
    """The 512^2 workload (sigma 20, 12x12 stride 3, 256 atoms, L=5, 10
    iterations), reference-compatible mode, against the FP64 oracle."""
    w = synth.WORKLOADS["img512_p12s3_k256"]
    clean, noisy = w.images()
    kw = dict(patch_width_dim=12, patch_height_dim=12, sliding_width=3, sliding_height=3, atoms=256, omp_iter=5,
              ksvd_iter=10, compat=3, precision=precision)
    with mkctx(ksvd, **kw) as c:
        out, st = c.denoise(noisy, w.sigma ** 2)
    ref, _ = oracle.ksvd_denoise(noisy, w.sigma ** 2, pw=12, ph=12, sw=3, sh=3, atoms=256, ksvd_iter=10,
                                 omp_iter=5, q1_cap=True, int_norm=True)
    pg, pr = synth.psnr(clean, out), synth.psnr(clean, ref)
    assert abs(pg - pr) <= 0.05, (pg, pr)


@pytest.mark.parametrize("precision", [0, 2])
def test_denoise_subimages_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, precision):
    """Sub-image mode: a 128 (x) x 100 (y) image cut into 60 x 48 sub-images
    (2 x 2 of them), each denoised with its own dictionary; the 8-pixel strip
    at the right and the 4 rows at the bottom are outside every sub-image and
    come back unchanged.  PSNR within 0.05 dB of the FP64 oracle."""
    clean = synth.clean_image(128, 51)[:100, :]
    noisy = synth.add_gaussian(clean, 20.0, 51)
    kw = dict(patch_width_dim=8, patch_height_dim=8, sliding_width=2, sliding_height=2, atoms=64, omp_iter=5,
              ksvd_iter=2, compat=1, precision=precision, sub_image_width_dim=48, sub_image_height_dim=60)
    with mkctx(ksvd, **kw) as c:
        out, st = c.denoise(noisy, 400.0)
    ref, lam = oracle.ksvd_denoise_tiled(noisy, 400.0, 48, 60, pw=8, ph=8, sw=2, sh=2, atoms=64, ksvd_iter=2,
                                         omp_iter=5, q1_cap=False, int_norm=True)
    np.testing.assert_array_equal(out[:, 120:], noisy[:, 120:])
    np.testing.assert_array_equal(out[96:, :], noisy[96:, :])
    pg, pr = synth.psnr(clean[:96, :120], out[:96, :120]), synth.psnr(clean[:96, :120], ref[:96, :120])
    assert abs(pg - pr) <= 0.05, (pg, pr)
    assert pg > synth.psnr(clean[:96, :120], noisy[:96, :120]) + 2.0
    assert st["num_patches"] == 4 * 27 * 21
    assert st["lambda_"] == pytest.approx(lam, rel=1e-2)


def test_subimage_errors(torch_cuda, ksvd, synth):
    img = synth.clean_image(64, 2)
    with mkctx(ksvd, atoms=16, sub_image_width_dim=80, sub_image_height_dim=32) as c:
        with pytest.raises(ksvd.KsvdError) as e:
            c.denoise(img, 100.0)
        assert e.value.status == ksvd.ERR_INVALID


@pytest.mark.parametrize("precision", [0, 2])
def test_denoise_rectangular_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, precision):
    """Rectangular patches on a non-square image: 5 (along y) x 7 (along x)
    patches at steps 3 (y) and 2 (x) on a 128 (x) x 100 (y) image, 48 atoms,
    L = 4, 3 iterations; PSNR within 0.05 dB of the FP64 oracle with the same
    (consistent) geometry."""
    clean = synth.clean_image(128, 61)[:100, :]
    noisy = synth.add_gaussian(clean, 20.0, 61)
    kw = dict(patch_width_dim=5, patch_height_dim=7, sliding_width=3, sliding_height=2, atoms=48, omp_iter=4,
              ksvd_iter=3, compat=1, precision=precision)
    with mkctx(ksvd, **kw) as c:
        out, st = c.denoise(noisy, 400.0)
    ref, info = oracle.ksvd_denoise(noisy, 400.0, pw=5, ph=7, sw=3, sh=2, atoms=48, ksvd_iter=3, omp_iter=4,
                                    q1_cap=False, int_norm=True)
    pg, pr = synth.psnr(clean, out), synth.psnr(clean, ref)
    assert abs(pg - pr) <= 0.05, (pg, pr)
    assert pg > synth.psnr(clean, noisy) + 1.0
    assert st["num_patches"] == oracle.num_patches(128, 100, 5, 7, 3, 2)


def test_build_image_rectangular_vs_oracle(torch_cuda, ksvd, oracle, synth):
    """createImage with 5 x 7 patches (steps 3 x 2) on a 128 x 100 image: the
    rebuilt pixels within 1e-5 relative of the oracle, lambda within 1e-5."""
    img = synth.add_gaussian(synth.clean_image(128, 62)[:100, :], 20.0, 62)
    Y = oracle.extract_patches(img, 5, 7, 3, 2)
    D = oracle.init_dictionary(Y, 24, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, 3, dtype=np.float32)
    c = mkctx(ksvd, patch_width_dim=5, patch_height_dim=7, sliding_width=3, sliding_height=2, atoms=24, omp_iter=3)
    out = torch_cuda.empty(img.shape, dtype=torch_cuda.float32, device="cuda")
    lam = c.build_image(dev(torch_cuda, img), 400.0, dev(torch_cuda, D), dev(torch_cuda, idx), dev(torch_cuda, coef),
                        out)
    ref, rlam = oracle.build_image(img, 5, 7, 3, 2, D, idx, coef, 400.0, dtype=np.float32)
    assert lam == pytest.approx(rlam, rel=1e-5)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-5, atol=1e-3)


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("shape", [(12, 3, 128), (16, 2, 320)])
def test_fused_residual_matches_separate_pass(torch_cuda, ksvd, synth, precision, shape):
    """Inside ksvd_iterate the OMP writes the update sweep's residual rows
    itself (the 16-bit form for patches that took L atoms, the residual
    kernel forming the rest; the FP32 form from its own residual tile; 320
    atoms of 16 x 16 take the streamed-dictionary kernels).  The same
    iteration through ksvd_omp and
    ksvd_update_dictionary, where the residual kernel forms every row, must
    give the same dictionary and codes bit for bit.  A zero block makes some
    patches stop after one atom, so both kinds of rows are exercised."""
    clean = synth.clean_image(160, 31)
    noisy = synth.add_gaussian(clean, 20.0, 31).astype(np.float32)
    noisy[0:36, 0:36] = 0.0  # away from the middle patches that seed the dictionary
    pw, st, K = shape
    kw = dict(patch_width_dim=pw, patch_height_dim=pw, sliding_width=st, sliding_height=st, atoms=K, omp_iter=5,
              precision=precision, compat=1)
    c = mkctx(ksvd, **kw)
    N = ksvd.num_patches(c.params, 160, 160)
    Y = torch_cuda.empty((N, c.n), dtype=torch_cuda.float32, device="cuda")
    c.extract_patches(dev(torch_cuda, noisy), Y)
    D0 = torch_cuda.empty((c.K, c.n), dtype=torch_cuda.float32, device="cuda")
    c.init_dictionary(Y, D0)
    out = []
    for fused in (True, False):
        D = D0.clone()
        idx = torch_cuda.empty((N, c.L), dtype=torch_cuda.int32, device="cuda")
        coef = torch_cuda.empty((N, c.L), dtype=torch_cuda.float32, device="cuda")
        for _ in range(2):
            if fused:
                c.iterate(Y, D, idx, coef, 1)
            else:
                c.omp(Y, D, idx, coef)
                c.update_dictionary(Y, D, idx, coef)
        torch_cuda.cuda.synchronize()
        out.append((D.cpu().numpy(), idx.cpu().numpy(), coef.cpu().numpy()))
    (Df, If, Cf), (Ds, Is, Cs) = out
    assert np.count_nonzero(If[:, 1] < 0) > 0  # some patches stopped after one atom
    assert np.array_equal(If, Is)
    assert np.array_equal(Cf.view(np.uint32), Cs.view(np.uint32))
    assert np.array_equal(Df.view(np.uint32), Ds.view(np.uint32))
