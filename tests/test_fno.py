"""FNO surrogate: device forward and hand-written backward against an FP64
PyTorch CPU reference of the same network; training reduces the loss."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

S, M, LAYERS = 32, 4, 2


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("S,M,LAYERS", [(S, M, LAYERS), (128, 16, 2)])
def test_fno_forward_and_gradients_match_fp64_reference(S, M, LAYERS):
    """Small grid (CUDA-core channel kernels, one partial pixel tile per row)
    and a 128 grid (tcgen05 channel GEMMs in the forward and the backward,
    BF16 operands; the full 16 retained modes)."""
    import torch
    from highuvlith_b200.fno import FnoSurrogate
    from oracle import fno_ref
    net = FnoSurrogate(grid=S, modes=M, layers=LAYERS, seed=7)
    rng = np.random.default_rng(3)
    masks = (rng.random((2, S, S)) > 0.5).astype(np.float32)
    targets = rng.random((2, S, S)).astype(np.float32)
    params = net.get_params()
    dm = torch.from_numpy(masks).cuda()
    out = net.forward(dm).cpu().numpy()
    net.device_status()  # no bounded device-side wait gave up
    ref, p, a = fno_ref.forward(params.astype(np.float64), masks, S, m=M, L=LAYERS, requires_grad=True)
    assert _rel(out, ref.detach().numpy()) < 2e-2
    # gradients of the MSE loss
    loss_ref = ((ref - torch.tensor(targets, dtype=torch.float64)) ** 2).mean()
    loss_ref.backward()
    loss, pg, ig = net.backward(dm, targets=torch.from_numpy(targets).cuda(), want_input_grad=True)
    assert abs(loss - loss_ref.item()) < 2e-2 * loss_ref.item()
    g_ref = p.grad.numpy()
    g = pg.cpu().numpy()
    assert _rel(g, g_ref) < 5e-2
    cos = float(np.dot(g, g_ref) / (np.linalg.norm(g) * np.linalg.norm(g_ref)))
    assert cos > 0.999
    assert _rel(ig.cpu().numpy(), a.grad.numpy()) < 5e-2


def test_fno_training_reduces_loss():
    import torch
    from highuvlith_b200.fno import FnoSurrogate
    net = FnoSurrogate(grid=S, modes=M, layers=LAYERS, seed=1)
    rng = np.random.default_rng(5)
    masks = torch.from_numpy((rng.random((4, S, S)) > 0.5).astype(np.float32)).cuda()
    # a smooth target the operator can represent: a blurred copy of the mask
    k = torch.fft.fft2(masks)
    f = torch.fft.fftfreq(S, device="cuda")
    g = torch.exp(-(f[:, None] ** 2 + f[None, :] ** 2) * 60.0)
    targets = torch.fft.ifft2(k * g).real.float().contiguous()
    losses = [net.train_step(masks, targets, lr=3e-3) for _ in range(60)]
    assert losses[-1] < 0.3 * losses[0], (losses[0], losses[-1])
