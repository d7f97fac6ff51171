"""ksvd_denoise_many: images of uneven size and patch shape (Gaussian and
speckle) through one pipeline, the atom sweeps of all images in one
persistent launch with the SMs split between them, iterations replayed from
a CUDA graph.  Per image: PSNR within 0.05 dB of the FP64 oracle, and close
to the one-image path (the split changes only the summation order of the
sweep's partial sums)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _jobs(ksvd, synth):
    spec = [  # side, patch, stride, speckle, sigma, precision
        (96, 8, 2, False, 20.0, 0),
        (128, 12, 3, False, 25.0, 2),
        (64, 6, 2, False, 15.0, 0),
        (112, 8, 3, True, None, 0),
        (160, 12, 3, False, 30.0, 1),
        (80, 10, 2, False, 35.0, 2),
    ]
    out = []
    for i, (side, patch, stride, speckle, sigma, prec) in enumerate(spec):
        clean = synth.clean_image(side, 70 + i)
        if speckle:
            clean = clean + 1.0
            noisy = synth.add_speckle(clean, 4.0, 70 + i)
            sigma2 = 0.3
        else:
            noisy = synth.add_gaussian(clean, sigma, 70 + i)
            sigma2 = sigma * sigma
        params = ksvd.make_params(patch_width_dim=patch, patch_height_dim=patch, sliding_width=stride,
                                  sliding_height=stride, atoms=48, omp_iter=4, ksvd_iter=3, speckle=int(speckle),
                                  compat=1, precision=prec)
        out.append(dict(params=params, clean=clean, noisy=noisy, sigma2=sigma2, patch=patch, stride=stride,
                        speckle=speckle))
    return out


@pytest.mark.parametrize("tune", [False, True])
def test_denoise_many_vs_oracle_and_single(torch_cuda, ksvd, oracle, synth, tune):
    jobs = _jobs(ksvd, synth)
    outs, st = ksvd.denoise_many([(j["params"], j["noisy"], j["sigma2"]) for j in jobs], tune=tune)
    assert st["graph"] == 1, st
    # the sweep's lanes: disjoint CTA ranges tiling the grid, every image in one
    sms = torch_cuda.cuda.get_device_properties(0).multi_processor_count
    lanes = {}
    for b, c in zip(st["update_cta_begin"], st["update_ctas"]):
        assert c >= 1 and 0 <= b and b + c <= sms
        lanes.setdefault(b, set()).add(c)
    assert all(len(w) == 1 for w in lanes.values()) and len(lanes) == st["lanes"]
    assert sum(next(iter(w)) for w in lanes.values()) == sms
    for j, out in zip(jobs, outs):
        p = j["patch"]
        ref, _ = oracle.ksvd_denoise(j["noisy"], j["sigma2"], pw=p, ph=p, sw=j["stride"], sh=j["stride"], atoms=48,
                                     ksvd_iter=3, omp_iter=4, speckle=j["speckle"], q1_cap=False, int_norm=True)
        assert np.all(np.isfinite(out))
        pg, pr = synth.psnr(j["clean"], out), synth.psnr(j["clean"], ref)
        assert abs(pg - pr) <= 0.05, (p, j["speckle"], pg, pr)
        with ksvd.Context(j["params"]) as c:
            single, _ = c.denoise(j["noisy"], j["sigma2"])
        assert abs(synth.psnr(j["clean"], single) - pg) <= 0.02


def test_denoise_many_rejects(torch_cuda, ksvd, synth):
    img = synth.clean_image(64, 1)
    p1 = ksvd.make_params(atoms=16, ksvd_iter=2)
    p2 = ksvd.make_params(atoms=16, ksvd_iter=3)
    with pytest.raises(ksvd.KsvdError) as e:
        ksvd.denoise_many([(p1, img, 100.0), (p2, img, 100.0)])  # different iteration counts
    assert e.value.status == ksvd.ERR_INVALID
    p3 = ksvd.make_params(atoms=16, ksvd_iter=2, precision=ksvd.PREC_BF16_LEARNED)
    with pytest.raises(ksvd.KsvdError):
        ksvd.denoise_many([(p3, img, 100.0)])
