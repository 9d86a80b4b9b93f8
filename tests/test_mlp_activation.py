"""The learned form's activation silu_p (mapp_b200/csrc/mg_mlp_common.cuh):
its stated error bounds against the exp-based SiLU, its derivative, and the
CUDA coefficients against the CPU reference's (tests/mlp_reference.py)."""
import os
import re

import numpy as np

from tests import mlp_reference as ref

HERE = os.path.dirname(os.path.abspath(__file__))


def test_sigma_and_silu_bounds():
    z = np.linspace(-80.0, 80.0, 1_600_001)
    sig = 1.0 / (1.0 + np.exp(-z))
    assert np.max(np.abs(ref.sigma_p(z) - sig)) <= 9.3e-4
    assert np.max(np.abs(ref.silu(z) - z * sig)) <= 6.4e-3
    # 0 and 1 beyond |z| = 7 (to the rounding of the coefficients), so
    # silu_p(z) vanishes for large negative z instead of growing with |z|
    assert np.all(ref.sigma_p(z[z <= -7.0]) <= 1e-6) and np.all(ref.sigma_p(z[z >= 7.0]) >= 1.0 - 1e-6)
    # FP32 evaluation (as the kernels run it) keeps the bound
    q32 = ref.SIG_Q.astype(np.float32)
    x = np.clip(z.astype(np.float32) * np.float32(1.0 / 7.0), -1, 1).astype(np.float32)
    u = x * x
    q = np.float32(q32[6])
    for k in range(5, -1, -1):
        q = (q * u + q32[k]).astype(np.float32)
    s32 = np.clip(x * q + np.float32(0.5), 0, 1).astype(np.float64)
    assert np.max(np.abs(s32 - sig)) <= 9.4e-4


def test_dsilu_is_the_derivative():
    z = np.linspace(-9.0, 9.0, 2001)
    h = 1e-5
    fd = (ref.silu(z + h) - ref.silu(z - h)) / (2 * h)
    assert np.max(np.abs(fd - ref.dsilu(z))) <= 1e-7


def test_cuda_coefficients_match_reference():
    src = open(os.path.join(HERE, "..", "mapp_b200", "csrc", "mg_mlp_common.cuh")).read()
    got = {int(k): float(v.rstrip("f")) for k, v in re.findall(r"kSigQ(\d) = ([-+0-9.e]+f)", src)}
    assert sorted(got) == list(range(7))
    assert np.allclose([got[k] for k in range(7)], ref.SIG_Q, rtol=0, atol=0)
