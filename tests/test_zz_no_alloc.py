"""ksvd_omp_noalloc, the OMP entry point for callers that cannot allocate
device memory (inside CUDA graph capture, under a framework that owns all
device allocations, in loops that must not allocate).  It keeps the
dictionary Gram in an array compiled into the library instead of context
memory; its results must match ksvd_omp's.  This file is collected last so a
run that stops at the first failure has run everything else first."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(oracle, synth, seed, K):
    img = synth.add_gaussian(synth.clean_image(96, seed), 20.0, seed)
    Y = oracle.extract_patches(img, 8, 8, 2, 2)
    D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
    return Y, D


def test_noalloc_matches_context_omp_twice(torch_cuda, ksvd, oracle, synth):
    torch = torch_cuda
    params = ksvd.make_params(patch_width_dim=8, patch_height_dim=8, sliding_width=2, sliding_height=2, atoms=64,
                              omp_iter=5, precision=ksvd.PREC_FP32)
    ctx = ksvd.Context(params)
    # two calls in a row with different inputs: the shared Gram array must be
    # fully rewritten by the second call
    for seed in (3, 4):
        Y, D = _case(oracle, synth, seed, 64)
        Yd, Dd = torch.from_numpy(Y).cuda(), torch.from_numpy(D).cuda()
        N = Y.shape[0]
        i1 = torch.empty((N, 5), dtype=torch.int32, device="cuda")
        c1 = torch.empty((N, 5), dtype=torch.float32, device="cuda")
        i2 = torch.full((N, 5), -7, dtype=torch.int32, device="cuda")
        c2 = torch.full((N, 5), 99.0, dtype=torch.float32, device="cuda")
        ctx.omp(Yd, Dd, i1, c1)
        torch.cuda.synchronize()
        st = ksvd.omp_noalloc(params, Yd, Dd, i2, c2)
        torch.cuda.synchronize()
        assert st == ksvd.OK
        # same support agreement / coefficient tolerance as the other OMP tests
        agree = float(np.mean(np.all(i1.cpu().numpy() == i2.cpu().numpy(), axis=1)))
        assert agree >= 0.999, agree
        np.testing.assert_allclose(c2.cpu().numpy(), c1.cpu().numpy(), rtol=1e-4, atol=1e-4)
    ctx.close()


def test_noalloc_rejects_too_many_atoms(torch_cuda, ksvd):
    torch = torch_cuda
    params = ksvd.make_params(patch_width_dim=4, patch_height_dim=4, atoms=513, omp_iter=2)
    Y = torch.zeros((600, 16), device="cuda")
    D = torch.zeros((513, 16), device="cuda")
    idx = torch.empty((600, 2), dtype=torch.int32, device="cuda")
    coef = torch.empty((600, 2), device="cuda")
    assert ksvd.omp_noalloc(params, Y, D, idx, coef) == ksvd.ERR_TOO_LARGE
