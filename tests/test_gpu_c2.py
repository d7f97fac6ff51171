"""The 2048^2 headline workload (sigma 25, 12 x 12 patches at stride 3,
461,041 patches, 256 atoms, L = 5, 10 iterations, full update without the
1024-patch cap) against the FP64 oracle, for every arithmetic form:

* first OMP call from the shared FP32 initial dictionary: ordered support
  agreement >= 99.9% and coefficients within 1e-4 of the patch's largest;
* first update sweep from the FP64 oracle's codes: every atom within 1e-4
  (relative, up to sign) and coefficients within 1e-4 of the patch's largest;
* the whole denoise (10 iterations, final OMP, rebuild): PSNR within 0.05 dB
  of the FP64 oracle's.

The FP64 reference (about a minute of CPU on 16 threads) is computed once."""

import numpy as np
import pytest

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

WORKLOAD = "img2048_p12s3_k256"
FORMS = {"fp32": 0, "bf16": 1, "fp16": 2}


@pytest.fixture(scope="module")
def quality():
    from ksvd_loader import load_oracle
    load_oracle()
    import quality as q
    return q


@pytest.fixture(scope="module")
def c2(torch_cuda, ksvd, oracle, synth, quality):
    torch = torch_cuda
    w = synth.WORKLOADS[WORKLOAD]
    clean, noisy = w.images()
    params = ksvd.make_params(patch_width_dim=w.patch, patch_height_dim=w.patch, sliding_width=w.stride,
                              sliding_height=w.stride, atoms=w.atoms, omp_iter=w.omp_iter, ksvd_iter=w.ksvd_iter,
                              compat=ksvd.COMPAT_INT_NORM)
    with ksvd.Context(params) as c:
        N = ksvd.num_patches(params, w.size, w.size)
        Yd = torch.empty((N, w.n), dtype=torch.float32, device="cuda")
        Dd = torch.empty((w.atoms, w.n), dtype=torch.float32, device="cuda")
        c.extract_patches(torch.from_numpy(noisy).cuda(), Yd)
        c.init_dictionary(Yd, Dd)
        torch.cuda.synchronize()
        D0 = Dd.cpu().numpy()
    ref = quality.fp64_reference(oracle, noisy, D0, patch=w.patch, stride=w.stride, omp_iter=w.omp_iter,
                                 ksvd_iter=w.ksvd_iter, q1_cap=False, sigma2=w.sigma ** 2)
    np.testing.assert_array_equal(Yd.cpu().numpy(), ref["Y"])
    return {"w": w, "clean": clean, "noisy": noisy, "D0": D0, "Yd": Yd, "ref": ref,
            "psnr64": synth.psnr(clean, ref["image"])}


def _ctx(ksvd, w, precision):
    return ksvd.Context(ksvd.make_params(patch_width_dim=w.patch, patch_height_dim=w.patch, sliding_width=w.stride,
                                         sliding_height=w.stride, atoms=w.atoms, omp_iter=w.omp_iter,
                                         ksvd_iter=w.ksvd_iter, compat=ksvd.COMPAT_INT_NORM, precision=precision))


@pytest.mark.parametrize("form", list(FORMS))
def test_c2_first_omp_vs_fp64(torch_cuda, ksvd, quality, c2, form):
    torch, w, ref = torch_cuda, c2["w"], c2["ref"]
    N = c2["Yd"].shape[0]
    idx = torch.empty((N, w.omp_iter), dtype=torch.int32, device="cuda")
    coef = torch.empty((N, w.omp_iter), dtype=torch.float32, device="cuda")
    with _ctx(ksvd, w, FORMS[form]) as c:
        c.omp(c2["Yd"], torch.from_numpy(c2["D0"]).cuda(), idx, coef)
        torch.cuda.synchronize()
    i, cf = idx.cpu().numpy(), coef.cpu().numpy()
    agree = quality.support_agreement(i, ref["idx0"])
    err = quality.coef_rel_err(i, cf, ref["idx0"], ref["coef0"])
    assert agree >= 0.999, (form, agree)
    assert err <= 1e-4, (form, err)


def test_c2_first_sweep_vs_fp64(torch_cuda, ksvd, quality, c2):
    torch, w, ref = torch_cuda, c2["w"], c2["ref"]
    Dd = torch.from_numpy(c2["D0"].copy()).cuda()
    idx = torch.from_numpy(ref["idx0"]).cuda()
    coef = torch.from_numpy(ref["coef0"].astype(np.float32)).cuda()
    with _ctx(ksvd, w, 0) as c:
        c.update_dictionary(c2["Yd"], Dd, idx, coef)
        torch.cuda.synchronize()
    a_err = quality.atom_err(Dd.cpu().numpy(), ref["D1"])
    c_err = quality.coef_rel_err(ref["idx0"], coef.cpu().numpy(), ref["idx0"], ref["coef1"])
    assert a_err <= 1e-4, a_err
    assert c_err <= 1e-4, c_err


@pytest.mark.parametrize("form", list(FORMS))
def test_c2_denoise_psnr_vs_fp64(ksvd, synth, c2, form):
    w = c2["w"]
    with _ctx(ksvd, w, FORMS[form]) as c:
        out, _ = c.denoise(c2["noisy"], w.sigma ** 2)
    p = synth.psnr(c2["clean"], out)
    assert abs(p - c2["psnr64"]) <= 0.05, (form, p, c2["psnr64"])
