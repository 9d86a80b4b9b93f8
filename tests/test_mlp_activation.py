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
    assert np.max(np.abs(ref.sigma_p(z) - sig)) <= 9.2e-4
    assert np.max(np.abs(ref.silu(z) - z * sig)) <= 7.3e-3
    # 0 and 1 beyond |z| = 8 (to the rounding of the coefficients), so
    # silu_p(z) vanishes for large negative z instead of growing with |z|
    assert np.all(ref.sigma_p(z[z <= -8.0]) <= 1e-7) and np.all(ref.sigma_p(z[z >= 8.0]) >= 1.0 - 1e-7)
    # FP32 evaluation (as the kernels run it, on x = z / 8) keeps the bound
    q32 = ref.SIG_Q.astype(np.float32)
    x = (z.astype(np.float32) * np.float32(0.125)).astype(np.float32)
    u = np.minimum(x * x, np.float32(1.0)).astype(np.float32)
    q = np.float32(q32[-1])
    for k in range(len(q32) - 2, -1, -1):
        q = (q * u + q32[k]).astype(np.float32)
    s32 = np.clip(x * q + np.float32(0.5), 0, 1).astype(np.float64)
    assert np.max(np.abs(s32 - sig)) <= 9.3e-4


def test_dsilu_is_the_derivative():
    z = np.linspace(-9.0, 9.0, 2001)
    # away from the two points where the clamp of sigma_p sets in
    su = 0.5 + (z / ref.SIG_Z) * np.polynomial.polynomial.polyval(np.minimum((z / ref.SIG_Z) ** 2, 1.0), ref.SIG_Q)
    z = z[(np.abs(su) > 1e-4) & (np.abs(su - 1.0) > 1e-4) & (np.abs(np.abs(z) - ref.SIG_Z) > 1e-3)]
    h = 1e-5
    fd = (ref.silu(z + h) - ref.silu(z - h)) / (2 * h)
    assert np.max(np.abs(fd - ref.dsilu(z))) <= 1e-7


def test_cuda_coefficients_match_reference():
    src = open(os.path.join(HERE, "..", "mapp_b200", "csrc", "mg_mlp_common.cuh")).read()
    got = {int(k): float(v.rstrip("f")) for k, v in re.findall(r"kSigQ(\d) = ([-+0-9.e]+f)", src)}
    n = len(ref.SIG_Q)
    assert sorted(got) == list(range(n))
    assert np.allclose([got[k] for k in range(n)], ref.SIG_Q, rtol=0, atol=0)
    assert int(re.search(r"kSplitTanh = (\d+);", src).group(1)) == ref.SPLIT_TANH


def test_split_activation_units():
    z = np.linspace(-6.0, 6.0, 64)[None, :].repeat(3, 0)
    a = ref.act(z, 2)
    assert np.array_equal(a[:, :ref.SPLIT_TANH], ref.silu_exact(z[:, :ref.SPLIT_TANH]))
    assert np.array_equal(a[:, ref.SPLIT_TANH:], ref.silu(z[:, ref.SPLIT_TANH:]))
