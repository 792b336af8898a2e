"""GPU tests of the tensor-core (tcgen05) MLP kernels against an FP64 reference
that applies the same BF16 rounding of weights, inputs and activations."""
import numpy as np
import pytest

from bcc import mlp

pytestmark = pytest.mark.gpu


def test_mlp_forward_matches_reference(checker):
    import torch
    rng = np.random.default_rng(0)
    p = mlp.init_params(1)
    P = mlp.unflatten(p)
    P["b1"][:] = rng.normal(0, 0.1, 128)
    P["b2"][:] = rng.normal(0, 0.1, 128)
    P["b3"][:] = rng.normal(0, 0.1, 128)
    P["b4"][:] = 0.3
    checker.mlp_set_params(p)
    for rows in (1, 128, 333, 5000):
        x = rng.normal(0, 1, (rows, 48)).astype(np.float32)
        x[:, 39:] = 0
        xb = torch.from_numpy(mlp.to_bf16_bits(x).view(np.int16)).cuda()
        out = torch.zeros(rows, dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        checker.mlp_forward_device(xb.data_ptr(), rows, out.data_ptr(), stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = mlp.forward_reference(p, x)
        scale = np.abs(want).max() + 1.0
        err = np.abs(got - want).max() / scale
        assert err < 2e-2, (rows, err)
    assert np.allclose(checker.mlp_get_params(), p)
