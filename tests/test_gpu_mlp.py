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


def test_mlp_gradients_match_cpu_oracle(checker):
    """Tensor-core training kernel gradients vs the FP64 CPU oracle."""
    import torch
    from oracle import mlp_oracle
    rng = np.random.default_rng(3)
    p = mlp.init_params(4)
    P = mlp.unflatten(p)
    for b in ("b1", "b2", "b3"):
        P[b][:] = rng.normal(0, 0.05, 128)
    checker.mlp_set_params(p)
    for rows in (77, 300, 2000):
        x = rng.normal(0, 1, (rows, 48)).astype(np.float32)
        x[:, 39:] = 0
        y = (rng.uniform(0, 1, rows) < 0.4).astype(np.uint8)
        xb = torch.from_numpy(mlp.to_bf16_bits(x).view(np.int16)).cuda()
        yb = torch.from_numpy(y).cuda()
        torch.cuda.synchronize()
        g, loss = checker.mlp_gradients_device(xb.data_ptr(), yb.data_ptr(), rows)
        want_loss, want = mlp_oracle.loss_and_grads(p, x, y)
        assert abs(loss - want_loss) < 1e-2 * want_loss + 1e-3, (loss, want_loss)
        o = 0
        for name, shape in mlp.SHAPES:
            k = int(np.prod(shape))
            a, b = g[o:o + k], want[o:o + k]
            rel = np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-12)
            assert rel < 3e-2, (rows, name, rel)
            o += k


def test_mlp_training_reduces_loss(checker):
    """A few Adam steps on a learnable synthetic rule lower the loss."""
    import torch
    rng = np.random.default_rng(5)
    checker.mlp_set_params(mlp.init_params(6))
    rows = 4096
    x = rng.normal(0, 1, (rows, 48)).astype(np.float32)
    x[:, 39:] = 0
    y = ((x[:, 0] + 0.5 * x[:, 3] - x[:, 10]) > 0.2).astype(np.uint8)
    xb = torch.from_numpy(mlp.to_bf16_bits(x).view(np.int16)).cuda()
    yb = torch.from_numpy(y).cuda()
    losses = [checker.mlp_train_step_device(xb.data_ptr(), yb.data_ptr(), rows, 3e-3) / rows for _ in range(60)]
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
