"""Dictionaries and patches beyond the shared-memory-resident OMP kernels:
512 atoms of 16x16 patches (the 4096^2 workload's shape) and 22x22 patches,
through the C ABI against the FP64 oracle.  Same bars as test_gpu_parity.py:
OMP support agreement >= 99.9% with coefficients within 1e-4 relative, atoms
within 1e-4, denoised PSNR within 0.05 dB."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def mkctx(ksvd, **kw):
    return ksvd.Context(ksvd.make_params(**kw))


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_omp(torch, ksvd, Y, D, **kw):
    c = mkctx(ksvd, **kw)
    N = Y.shape[0]
    idx = torch.empty((N, c.L), dtype=torch.int32, device="cuda")
    coef = torch.empty((N, c.L), dtype=torch.float32, device="cuda")
    c.omp(dev(torch, Y), dev(torch, D), idx, coef)
    torch.cuda.synchronize()
    return idx.cpu().numpy(), coef.cpu().numpy()


def check_omp(idx, coef, ri, rc):
    agree = float(np.mean(np.all(idx == ri, axis=1)))
    assert agree >= 0.999, agree
    m = np.all(idx == ri, axis=1)
    rel = np.abs(coef[m] - rc[m]) / (np.abs(rc[m]).max(axis=1, keepdims=True) + 1e-30)
    assert rel.max() < 1e-4, rel.max()


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_omp_512_atoms_16x16(torch_cuda, ksvd, oracle, synth, precision):
    """n = 256, K = 512, L = 8 (the 4096^2 workload's dictionary shape): the
    FP32 form streams the dictionary through shared memory; the 16-bit forms
    stream 16-feature slices of the 16-bit dictionary through a ring of
    shared-memory slots into 512 TMEM columns (kernels_omp_tcb.cu)."""
    noisy = synth.add_gaussian(synth.clean_image(128, 41), 15.0, 41)
    Y = oracle.extract_patches(noisy, 16, 16, 2, 2)
    D = oracle.init_dictionary(Y, 512, int_norm=True, dtype=np.float32)
    idx, coef = run_omp(torch_cuda, ksvd, Y, D, patch_width_dim=16, patch_height_dim=16, sliding_width=2,
                        sliding_height=2, atoms=512, omp_iter=8, precision=precision)
    ri, rc = oracle.omp(Y.astype(np.float64), D.astype(np.float64), 8)
    check_omp(idx, coef, ri, rc)


@pytest.mark.parametrize("precision", [0, 2])
def test_omp_22x22_patches(torch_cuda, ksvd, oracle, synth, precision):
    """n = 484 (22x22 patches), K = 256, L = 5: FP32 with the dictionary
    streamed through shared memory, FP16 with the 16-bit dictionary streamed
    slice by slice (kernels_omp_tcb.cu)."""
    noisy = synth.add_gaussian(synth.clean_image(112, 42), 25.0, 42)
    Y = oracle.extract_patches(noisy, 22, 22, 3, 3)
    D = oracle.init_dictionary(Y, 256, int_norm=True, dtype=np.float32)
    idx, coef = run_omp(torch_cuda, ksvd, Y, D, patch_width_dim=22, patch_height_dim=22, sliding_width=3,
                        sliding_height=3, atoms=256, omp_iter=5, precision=precision)
    ri, rc = oracle.omp(Y.astype(np.float64), D.astype(np.float64), 5)
    check_omp(idx, coef, ri, rc)


def test_update_512_atoms_16x16(torch_cuda, ksvd, oracle, synth):
    noisy = synth.add_gaussian(synth.clean_image(128, 43), 15.0, 43)
    Y = oracle.extract_patches(noisy, 16, 16, 2, 2)
    K, L = 512, 8
    D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, L, dtype=np.float32)
    c = mkctx(ksvd, patch_width_dim=16, patch_height_dim=16, sliding_width=2, sliding_height=2, atoms=K,
              omp_iter=L, compat=1)
    Dd = dev(torch_cuda, D)
    cd = dev(torch_cuda, coef.astype(np.float32))
    c.update_dictionary(dev(torch_cuda, Y), Dd, dev(torch_cuda, idx), cd)
    torch_cuda.cuda.synchronize()
    Dr, cr = oracle.update_dictionary(Y.astype(np.float64), D.astype(np.float64), idx, coef.astype(np.float64),
                                      q1_cap=False)
    err = np.abs(Dd.cpu().numpy() - Dr).max()
    assert err < 1e-4, err
    assert np.abs(cd.cpu().numpy() - cr).max() < 1e-4 * np.abs(cr).max()


@pytest.mark.parametrize("pw,sw,K,L,size", [(16, 2, 512, 8, 96), (22, 3, 256, 5, 112)])
def test_denoise_large_shapes_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, pw, sw, K, L, size):
    clean = synth.clean_image(size, 44)
    noisy = synth.add_gaussian(clean, 15.0, 44)
    kw = dict(patch_width_dim=pw, patch_height_dim=pw, sliding_width=sw, sliding_height=sw, atoms=K, omp_iter=L,
              ksvd_iter=1, compat=1)
    with mkctx(ksvd, **kw) as c:
        out, _ = c.denoise(noisy, 225.0)
    ref, _ = oracle.ksvd_denoise(noisy, 225.0, pw=pw, ph=pw, sw=sw, sh=sw, atoms=K, ksvd_iter=1, omp_iter=L,
                                 q1_cap=False, int_norm=True)
    pg, pr = synth.psnr(clean, out), synth.psnr(clean, ref)
    assert abs(pg - pr) <= 0.05, (pg, pr)


@pytest.mark.parametrize("side,pw,K,speckle", [(96, 8, 64, False), (112, 12, 128, True), (128, 22, 64, False)])
def test_uneven_images_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, side, pw, K, speckle):
    """Images of the uneven multi-image workload's kinds (8x8, 12x12 and 22x22
    patches at stride 3, Gaussian or speckle noise), one context each, against
    the FP64 oracle."""
    clean = synth.clean_image(side, 60 + pw) + (1.0 if speckle else 0.0)
    noisy = synth.add_speckle(clean, 4.0, 60 + pw) if speckle else synth.add_gaussian(clean, 30.0, 60 + pw)
    sigma2 = 0.3 if speckle else 900.0
    kw = dict(patch_width_dim=pw, patch_height_dim=pw, sliding_width=3, sliding_height=3, atoms=K, omp_iter=5,
              ksvd_iter=1, compat=1, speckle=int(speckle))
    with mkctx(ksvd, **kw) as c:
        out, _ = c.denoise(noisy, sigma2)
    ref, _ = oracle.ksvd_denoise(noisy, sigma2, pw=pw, ph=pw, sw=3, sh=3, atoms=K, ksvd_iter=1, omp_iter=5,
                                 speckle=speckle, q1_cap=False, int_norm=True)
    assert np.all(np.isfinite(out))
    pg, pr = synth.psnr(clean, out), synth.psnr(clean, ref)
    assert abs(pg - pr) <= 0.05, (pg, pr)


def test_update_mixed_atom_sizes_deterministic(torch_cuda, ksvd, oracle, synth):
    """16x16 patches of an image that is flat outside a textured cross: three
    atoms carry more than 13,000 entries beside small ones; the largest has
    more than the sweep's CTAs hold in shared memory, so part of its columns
    stream from the residual on every pass.  Atoms and coefficients against
    the FP64 oracle (1e-4); two runs agree bit for bit."""
    S, K, L = 224, 32, 3
    tex = synth.add_gaussian(synth.clean_image(S, 70), 10.0, 70)
    img = np.full((S, S), 100.0, np.float32)
    img[88:136, :] = tex[88:136, :]
    img[:, 88:136] = tex[:, 88:136]
    Y = oracle.extract_patches(img, 16, 16, 1, 1)
    D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
    idx, coef = oracle.omp(Y, D, L, dtype=np.float32)
    cnt = np.bincount(idx[(idx >= 0) & (coef != 0)], minlength=K)
    assert (cnt > 13100).sum() >= 2 and (cnt < 5000).sum() >= 10, cnt
    c = mkctx(ksvd, patch_width_dim=16, patch_height_dim=16, sliding_width=1, sliding_height=1, atoms=K,
              omp_iter=L, compat=1)
    Yd, idd = dev(torch_cuda, Y), dev(torch_cuda, idx)
    runs = []
    for _ in range(2):
        Dd, cd = dev(torch_cuda, D), dev(torch_cuda, coef.astype(np.float32))
        c.profile(1)
        c.profile_reset()
        c.update_dictionary(Yd, Dd, idd, cd)
        torch_cuda.cuda.synchronize()
        cn = c.profile_counters()
        c.profile(0)
        runs.append((Dd.cpu().numpy(), cd.cpu().numpy()))
        assert cn["atoms_updated"] == K
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
    Dr, cr = oracle.update_dictionary(Y.astype(np.float64), D.astype(np.float64), idx, coef.astype(np.float64),
                                      q1_cap=False)
    err = np.abs(runs[0][0] - Dr).max()
    assert err < 1e-4, err
    assert np.abs(runs[0][1] - cr).max() < 1e-4 * np.abs(cr).max()


@pytest.mark.parametrize("precision", [1, 2])
def test_omp_tcb_shapes(torch_cuda, ksvd, oracle, synth, precision):
    """The streamed tensor-core kernel at other shapes it serves: 300 atoms
    of 12 x 12 patches (Kp = 304 columns, a partial last quarter), 400 atoms
    of 10 x 10 patches (n not a multiple of 16), fewer patches than a tile."""
    for side, patch, step, K, L, rows in ((96, 12, 3, 300, 5, None), (88, 10, 2, 400, 6, None),
                                          (96, 12, 3, 300, 5, 77)):
        noisy = synth.add_gaussian(synth.clean_image(side, 44 + K), 20.0, 44 + K)
        Y = oracle.extract_patches(noisy, patch, patch, step, step)
        D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
        if rows:
            Y = np.ascontiguousarray(Y[:rows])
        idx, coef = run_omp(torch_cuda, ksvd, Y, D, patch_width_dim=patch, patch_height_dim=patch,
                            sliding_width=step, sliding_height=step, atoms=K, omp_iter=L, precision=precision)
        ri, rc = oracle.omp(Y.astype(np.float64), D.astype(np.float64), L)
        check_omp(idx, coef, ri, rc)


@pytest.mark.slow
@pytest.mark.parametrize("precision", [0, 2])
def test_denoise_img4096_shape_vs_fp64_oracle(torch_cuda, ksvd, oracle, synth, precision):
    """The 4096^2 workload's settings (sigma 15, 16 x 16 patches at stride 2,
    512 atoms, L = 8, 8 iterations) on a 256^2 image of the same generator
    (14,641 patches): PSNR within 0.05 dB of the FP64 oracle."""
    w = synth.WORKLOADS["img4096_p16s2_k512"]
    clean = synth.clean_image(256, w.seed)
    noisy = synth.add_gaussian(clean, w.sigma, w.seed)
    kw = dict(patch_width_dim=16, patch_height_dim=16, sliding_width=2, sliding_height=2, atoms=512, omp_iter=8,
              ksvd_iter=8, compat=1, precision=precision)
    with mkctx(ksvd, **kw) as c:
        out, _ = c.denoise(noisy, w.sigma ** 2)
    ref, _ = oracle.ksvd_denoise(noisy, w.sigma ** 2, pw=16, ph=16, sw=2, sh=2, atoms=512, ksvd_iter=8, omp_iter=8,
                                 q1_cap=False, int_norm=True)
    pg, pr = synth.psnr(clean, out), synth.psnr(clean, ref)
    assert abs(pg - pr) <= 0.05, (pg, pr)
