"""The THINC face value of alpha1, face by face, against the reference's own host function.

The stage kernels compute the tanh profile of include/Operators_FV/Reconstruction2Face_THINC_D.H:13-35
with CUDA's exp, log and tanh, the reference's CPU build with the C library's; both are accurate to a
few ulps, not correctly rounded, so the face values can differ in the last bits, and that difference is
what the THINC runs amplify (tests/test_gpu_thinc.py). Here it is measured directly on 200 000 seeded
parameter sets over the ranges THINC uses (steepness beta = Beta (|n_d| + 0.01) in [0.02, 2.4] with the
default Beta 2.3, sign +-1, cell means in (EPS, 1 - EPS) with EPS 1e-4, both faces): the largest
difference and its distribution in ulps are printed, and bounded by 1e-13 absolute (alpha1 is in [0, 1]).
"""
import numpy as np
import pytest

import compas_b200 as cb
from oracle.oracle import have_ref, thinc_face_values

pytestmark = pytest.mark.gpu


def test_thinc_face_value_matches_the_reference_function():
    import torch

    if not have_ref(cb.SIXEQS, 3):
        pytest.skip("reference-header oracle not built")
    rng = np.random.default_rng(7)
    n = 200_000
    beta = 2.3 * (rng.uniform(0.0, 1.0, n) + 0.01)
    sigma = rng.choice([-1.0, 1.0], n)
    abar = rng.uniform(1e-4, 1.0 - 1e-4, n)
    side = rng.integers(0, 2, n).astype(np.int32)
    ref = thinc_face_values(beta, sigma, abar, side)
    dev = [torch.from_numpy(x).cuda() for x in (beta, sigma, abar, side)]
    out = torch.zeros(n, dtype=torch.float64, device="cuda")
    cb.thinc_face_values(*dev, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    diff = np.abs(got - ref)
    ulps = np.abs(got.view(np.int64) - ref.view(np.int64))
    frac_equal = float(np.mean(ulps == 0))
    print(f"THINC face values: {100 * frac_equal:.2f} % bit-identical, ulp differences max {int(ulps.max())}, "
          f"99.9th percentile {int(np.percentile(ulps, 99.9))}; max absolute difference {diff.max():.2e}")
    assert diff.max() <= 1e-13, diff.max()
