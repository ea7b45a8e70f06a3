"""GPU checks of the learned warm start's own kernels: conv3d forward, backward (weight,
bias and input gradients through the whole residual network), subspace channel packing,
and Adam training, against the FP64 CNN oracle with the same BF16-rounded weights."""
import numpy as np
import pytest

from conftest import rel_err
from oracle import cnn_oracle as CO

pytestmark = pytest.mark.gpu

CH = (14, 32, 32, 32, 32, 32, 32, 32, 14)


def _net(seed=1):
    from llr_b200.cnn import Cnn
    return Cnn(CH, seed=seed)


def test_forward_matches_oracle(gpu):
    rng = np.random.default_rng(5)
    x = rng.standard_normal((7, 6, 5, 14)).astype(np.float32)      # (nz, ny, nx, C), ragged tiles
    with _net() as net:
        p = net.params
        p[CO.layer_slices(CH)[0][0][1]:][:32] = rng.standard_normal(32) * 0.1   # non-zero biases
        net.params = p
        got = net.forward(x)
    exp, _ = CO.forward(p, CH, x.astype(np.float64))
    assert rel_err(got, exp) < 1e-5
    assert rel_err(got - x, exp - x) < 1e-4


@pytest.mark.parametrize("dims", [(4, 9, 10), (9, 8, 17)])
def test_gradients_match_oracle(gpu, dims):
    """dL/dW and dL/db of every layer for L = mean |out - target|^2."""
    from llr_b200.cnn import DeviceArray
    rng = np.random.default_rng(6)
    x = rng.standard_normal(dims + (14,)).astype(np.float32)
    t = rng.standard_normal(dims + (14,)).astype(np.float32)
    with _net(seed=2) as net:
        p = net.params
        dx, dt = DeviceArray.from_numpy(x), DeviceArray.from_numpy(t)
        loss = net.loss_grad_dev(dx, dt)
        g = net.grads
    el, eg = CO.loss_and_grads(p, CH, x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - el) <= 1e-5 * el
    for (w0, b0), co in zip(CO.layer_slices(CH)[0], CH[1:]):
        assert rel_err(g[w0:b0], eg[w0:b0]) < 1e-4
        assert rel_err(g[b0:b0 + co], eg[b0:b0 + co]) < 1e-4


def test_subspace_channels_and_image_match_oracle(gpu):
    import llr_b200
    from llr_b200 import DeviceBuffer
    from llr_b200.cnn import DeviceArray, subspace_channels_dev, subspace_image_dev
    rng = np.random.default_rng(7)
    vol, nq, r = (5, 6, 7), 11, 7
    S, _ = np.linalg.qr(rng.standard_normal((nq, r)) + 1j * rng.standard_normal((nq, r)))
    S = S.astype(np.complex64)
    x = (rng.standard_normal(vol + (nq,)) + 1j * rng.standard_normal(vol + (nq,))).astype(np.complex64)
    dx, dS = DeviceBuffer.from_array(x), DeviceBuffer.from_array(np.asfortranarray(S))
    ch = DeviceArray((vol[2], vol[1], vol[0], 2 * r))
    subspace_channels_dev(dx.ptr, vol, nq, dS.ptr, r, 3.0, ch)
    llr_b200._lib.check(llr_b200._lib.lib.llr_stream_sync(None))
    got = ch.numpy()
    assert rel_err(got, CO.subspace_channels(x.astype(np.complex128), S.astype(np.complex128), 3.0)) < 1e-6
    dy = DeviceBuffer(x.nbytes)
    subspace_image_dev(ch, vol, nq, dS.ptr, r, 3.0, dy.ptr)
    back = dy.download(np.empty_like(x, order="F"))
    assert rel_err(back, CO.subspace_image(got.astype(np.float64), S.astype(np.complex128), 3.0)) < 1e-6
    # demodulated by the unit phase u of a reference image: channels of u* x, image u (c S^H)
    ref = (rng.standard_normal(vol + (nq,)) + 1j * rng.standard_normal(vol + (nq,))).astype(np.complex64)
    ref[0, 0, 0, 0] = 0                                           # a zero reference maps to u = 1
    u = np.where(ref == 0, 1.0, ref / np.maximum(np.abs(ref), 1e-30))
    dref = DeviceBuffer.from_array(ref)
    subspace_channels_dev(dx.ptr, vol, nq, dS.ptr, r, 3.0, ch, dref.ptr)
    llr_b200._lib.check(llr_b200._lib.lib.llr_stream_sync(None))
    gotp = ch.numpy()
    assert rel_err(gotp, CO.subspace_channels(np.conj(u) * x.astype(np.complex128), S.astype(np.complex128), 3.0)) < 1e-6
    subspace_image_dev(ch, vol, nq, dS.ptr, r, 3.0, dy.ptr, d_phase_ref=dref.ptr)
    backp = dy.download(np.empty_like(x, order="F"))
    assert rel_err(backp, u * CO.subspace_image(gotp.astype(np.float64), S.astype(np.complex128), 3.0)) < 1e-6


def _adam_oracle(p, x, t, steps, lr, b1=0.9, b2=0.999, eps=1e-8):
    """FP64 Adam on the oracle's gradients, FP32 master weights rounded to BF16 in use."""
    p = p.astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    losses = []
    for k in range(1, steps + 1):
        loss, g = CO.loss_and_grads(p.astype(np.float32), CH, x, t)
        losses.append(loss)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        p = p - lr * (m / (1 - b1 ** k)) / (np.sqrt(v / (1 - b2 ** k)) + eps)
    return np.asarray(losses)


def test_adam_steps_match_oracle(gpu):
    """Five Adam steps on the GPU follow the oracle's loss trajectory."""
    from llr_b200.cnn import Cnn, DeviceArray
    rng = np.random.default_rng(8)
    x = rng.standard_normal((6, 8, 8, 14)).astype(np.float32)
    t = 0.5 * x
    with Cnn(CH, seed=12) as net:
        p0 = net.params
        dx, dt = DeviceArray.from_numpy(x), DeviceArray.from_numpy(t)
        got = np.asarray([net.train_step_dev(dx, dt, 2e-3) for _ in range(5)])
    exp = _adam_oracle(p0, x.astype(np.float64), t.astype(np.float64), 5, 2e-3)
    np.testing.assert_allclose(got, exp, rtol=2e-3)


def test_adam_training_reduces_loss(gpu):
    """Adam on the GPU kernels fits a damping map (target = 0.5 x: the residual branch must
    learn -0.5 x) on a 6 x 8 x 8 volume; the oracle reaches 1e-2 of the first loss in 50 steps."""
    from llr_b200.cnn import Cnn, DeviceArray
    rng = np.random.default_rng(8)
    x = rng.standard_normal((6, 8, 8, 14)).astype(np.float32)
    t = 0.5 * x
    with Cnn(CH, seed=12) as student:
        dx, dt = DeviceArray.from_numpy(x), DeviceArray.from_numpy(t)
        first = student.loss_grad_dev(dx, dt)
        for _ in range(100):
            last = student.train_step_dev(dx, dt, 2e-3)
    assert np.isfinite(last) and last < 0.05 * first, (first, last)


def test_learned_warm_start_gain(gpu):
    """Train on the GPU (own kernels) on adjoint -> converged pairs of 16 subjects that share
    one protocol, then start a held-out subject's recon from the network's image: it starts
    closer to the converged image than the zero-filled start, needs no more iterations to reach
    NRMSE <= 3e-2 and is no farther after 200 iterations (fixed partition, shared by both)."""
    from llr_b200 import warmstart as W
    from llr_b200.cnn import Cnn
    proto = W.Protocol(vol=(36, 36, 36), centre=9)      # 6^3 blocks tile the volume exactly
    codec = W.SubspaceCodec(proto)
    pairs = W.training_pairs(proto, codec, list(range(200, 216)), 400)
    with Cnn(seed=5) as net:
        losses = W.train(net, pairs, epochs=30, lr=1e-3)
        assert losses[-1] < 0.8 * losses[0]
        d = proto.subject(977)
        x_zf, x_ref, lam, energy, snap = W.reference(proto, d.y, 1600, snapshot=True)
        x0, ms = W.warm_start_image(net, codec, x_zf, energy, d.y)
    e_zf, e_ws = W.nrmse(x_zf, x_ref), W.nrmse(x0, x_ref)
    assert e_ws < e_zf, (e_ws, e_zf)
    plain, cp = W.time_to_targets(proto, d.y, lam, x_zf, snap, [3e-2, 1e-9], 200)
    learned, cl = W.time_to_targets(proto, d.y, lam, x0, snap, [3e-2, 1e-9], 200)
    assert abs(cp[0][1] - e_zf) < 1e-4 and abs(cl[0][1] - e_ws) < 1e-4   # device distance = host NRMSE
    assert plain[3e-2] is not None and learned[3e-2] is not None
    assert learned[3e-2][0] <= plain[3e-2][0], (learned, plain)
    assert cl[-1][1] <= cp[-1][1] * 1.05, (cl[-1], cp[-1])      # still at least as close after 200
