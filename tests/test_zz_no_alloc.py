"""ksvd_omp_noalloc, the OMP entry point for callers that cannot allocate
device memory (inside CUDA graph capture, under a framework that owns all
device allocations, in loops that must not allocate).  It keeps the
dictionary Gram in an array compiled into the library instead of context
memory and runs the same FP32 kernel as ksvd_omp, so its codes must equal
ksvd_omp's bit for bit.  This file is collected last so a run that stops at
the first failure has run everything else first."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(oracle, synth, seed, K, patch, step, side=96):
    img = synth.add_gaussian(synth.clean_image(side, seed), 20.0, seed)
    Y = oracle.extract_patches(img, patch, patch, step, step)
    D = oracle.init_dictionary(Y, K, int_norm=True, dtype=np.float32)
    return Y, D


def _compare(torch, ksvd, oracle, synth, K, patch, step, seeds, L=5):
    params = ksvd.make_params(patch_width_dim=patch, patch_height_dim=patch, sliding_width=step,
                              sliding_height=step, atoms=K, omp_iter=L, precision=ksvd.PREC_FP32)
    ctx = ksvd.Context(params)
    # calls in a row with different inputs: the shared Gram array must be
    # fully rewritten by each call
    for seed in seeds:
        Y, D = _case(oracle, synth, seed, K, patch, step)
        Yd, Dd = torch.from_numpy(Y).cuda(), torch.from_numpy(D).cuda()
        N = Y.shape[0]
        i1 = torch.empty((N, L), dtype=torch.int32, device="cuda")
        c1 = torch.empty((N, L), dtype=torch.float32, device="cuda")
        i2 = torch.full((N, L), -7, dtype=torch.int32, device="cuda")
        c2 = torch.full((N, L), 99.0, dtype=torch.float32, device="cuda")
        ctx.omp(Yd, Dd, i1, c1)
        torch.cuda.synchronize()
        st = ksvd.omp_noalloc(params, Yd, Dd, i2, c2)
        torch.cuda.synchronize()
        assert st == ksvd.OK
        # same kernel, same inputs: identical codes
        np.testing.assert_array_equal(i2.cpu().numpy(), i1.cpu().numpy())
        np.testing.assert_array_equal(c2.cpu().numpy(), c1.cpu().numpy())
    ctx.close()


def test_noalloc_matches_context_omp_twice(torch_cuda, ksvd, oracle, synth):
    _compare(torch_cuda, ksvd, oracle, synth, K=64, patch=8, step=2, seeds=(3, 4))


def test_noalloc_largest_dictionary(torch_cuda, ksvd, oracle, synth):
    """512 atoms, the largest the fixed array holds (8 x 8 patches)."""
    _compare(torch_cuda, ksvd, oracle, synth, K=512, patch=8, step=2, seeds=(5, 6))


def test_noalloc_streamed_dictionary(torch_cuda, ksvd, oracle, synth):
    """12 x 12 patches with 384 atoms: the FP32 dictionary (221 KB) does not
    fit in shared memory next to the tile, so both entry points stream it."""
    _compare(torch_cuda, ksvd, oracle, synth, K=384, patch=12, step=3, seeds=(7, 8))


def test_noalloc_rejects_too_many_atoms(torch_cuda, ksvd):
    torch = torch_cuda
    for patch in (4, 12):
        n = patch * patch
        params = ksvd.make_params(patch_width_dim=patch, patch_height_dim=patch, atoms=513, omp_iter=2)
        Y = torch.zeros((1200, n), device="cuda")
        D = torch.zeros((513, n), device="cuda")
        idx = torch.empty((1200, 2), dtype=torch.int32, device="cuda")
        coef = torch.empty((1200, 2), device="cuda")
        assert ksvd.omp_noalloc(params, Y, D, idx, coef) == ksvd.ERR_TOO_LARGE
