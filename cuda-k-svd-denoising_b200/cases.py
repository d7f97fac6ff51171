"""Small single-kernel runs of the library, for profilers (one case per
argument; each prints "ok <patches>" and exits 0):

  tcb       the 4096^2 workload's shape (16 x 16 patches at stride 2, 512
            atoms, L = 8) on a 1024^2 seeded image: three FP16 OMP calls, the
            tensor-core kernel with the streamed dictionary;
  proposal  the learned proposal's inference (three tcgen05 GEMM layers and
            the top-16 selection) on the 1536^2 image's 259,081 patches of
            144 values, random weights, twice.

Usage: python cuda-k-svd-denoising_b200/cases.py tcb|proposal
"""

from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def case_tcb():
    import torch
    from ksvd_loader import load
    pkg = load()
    ksvd = pkg.ksvd
    img = pkg.synth.add_gaussian(pkg.synth.clean_image(1024, 77), 15.0, 77)
    p = ksvd.make_params(patch_width_dim=16, patch_height_dim=16, sliding_width=2, sliding_height=2, atoms=512,
                         omp_iter=8, precision=ksvd.PREC_FP16_RESCORE)
    c = ksvd.Context(p)
    N = ksvd.num_patches(p, 1024, 1024)
    Y = torch.empty((N, 256), device="cuda")
    D = torch.empty((512, 256), device="cuda")
    c.extract_patches(torch.from_numpy(img).cuda(), Y)
    c.init_dictionary(Y, D)
    idx = torch.empty((N, 8), dtype=torch.int32, device="cuda")
    coef = torch.empty((N, 8), device="cuda")
    for _ in range(3):
        c.omp(Y, D, idx, coef)
    torch.cuda.synchronize()
    return N


def case_proposal():
    import torch
    from ksvd_loader import load
    pkg = load()
    ksvd = pkg.ksvd
    wl = pkg.synth.WORKLOADS["img1536_p12s3_k256"]
    _, noisy = wl.images()
    p = ksvd.make_params(patch_width_dim=12, patch_height_dim=12, sliding_width=3, sliding_height=3, atoms=256,
                         omp_iter=5, precision=ksvd.PREC_BF16_LEARNED)
    c = ksvd.Context(p)
    N = ksvd.num_patches(p, wl.size, wl.size)
    Y = torch.empty((N, 144), device="cuda")
    c.extract_patches(torch.from_numpy(noisy).cuda(), Y)
    c.proposal_init(3)
    cand = torch.empty((N, 16), dtype=torch.int32, device="cuda")
    for _ in range(2):
        c.proposal_candidates(Y, cand)
    torch.cuda.synchronize()
    return N


CASES = {"tcb": case_tcb, "proposal": case_proposal}

if __name__ == "__main__":
    if len(sys.argv) != 2 or sys.argv[1] not in CASES:
        sys.exit(__doc__)
    print("ok", CASES[sys.argv[1]]())
