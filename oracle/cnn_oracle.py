"""CPU oracle of the learned warm-start network (test infrastructure only).

FP64 numpy restatement of the 3-D residual CNN the library trains with its own kernels:
conv3d 3x3x3 with zero padding, ReLU between layers, out = in + net(in), mean-squared-error
loss, and the analytic backward pass (weight, bias and input gradients).  The reference has
no learned component, so nothing here is pinned to it: the oracle is pinned by a
finite-difference check of its own gradients (tests/test_cnn_oracle.py), and the GPU kernels
are checked against it with the same BF16-rounded weights.

Layouts match the device: activations (nz, ny, nx, C) C-order (voxel x fastest, channels
last); per layer W[27][cin][cout] with tap = dx + 3 (dy + 3 dz), then b[cout].

Warm-start training pairs (adjoint image -> converged recon) are built by the plain
recon itself; the subspace projection follows dti_subspace.rs:141-207 (c = x S, x = c S^H).
"""
from __future__ import annotations

import numpy as np


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def layer_slices(channels):
    """(W offset, b offset) per layer in the flat parameter vector."""
    out, off = [], 0
    for ci, co in zip(channels[:-1], channels[1:]):
        w = off
        off += 27 * ci * co
        out.append((w, off))
        off += co
    return out, off


def unpack(params: np.ndarray, channels, round_weights=True):
    """[(W (3,3,3,cin,cout) indexed [dz,dy,dx,ci,co], b (cout,))] from the flat vector."""
    sl, _ = layer_slices(channels)
    layers = []
    for (w, b), ci, co in zip(sl, channels[:-1], channels[1:]):
        W = params[w:w + 27 * ci * co].astype(np.float64)
        if round_weights:
            W = bf16_round(params[w:w + 27 * ci * co])
        layers.append((W.reshape(3, 3, 3, ci, co), params[b:b + co].astype(np.float64)))
    return layers


def conv3d(x: np.ndarray, W: np.ndarray, b) -> np.ndarray:
    """y[z,y,x,co] = b[co] + sum_{dz,dy,dx,ci} W[dz,dy,dx,ci,co] xpad[z+dz, y+dy, x+dx, ci]."""
    nz, ny, nx, _ = x.shape
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((nz, ny, nx, W.shape[4]))
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                y += xp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :] @ W[dz, dy, dx]
    if b is not None:
        y += b
    return y


def forward(params, channels, x, round_weights=True):
    """Returns (out, activations): activations[l] is the input of layer l."""
    layers = unpack(params, channels, round_weights)
    acts = [np.asarray(x, dtype=np.float64)]
    h = acts[0]
    for l, (W, b) in enumerate(layers):
        h = conv3d(h, W, b)
        if l + 1 < len(layers):
            h = np.maximum(h, 0.0)
            acts.append(h)
    return acts[0] + h, acts


def loss_and_grads(params, channels, x, target, round_weights=True):
    """Mean-squared-error loss and its gradient with respect to the flat parameter vector
    (through the BF16-rounded weights, as the GPU computes it, unless round_weights=False)."""
    layers = unpack(params, channels, round_weights)
    out, acts = forward(params, channels, x, round_weights)
    n = out.size
    loss = float(np.mean((out - target) ** 2))
    g = 2.0 * (out - target) / n
    sl, total = layer_slices(channels)
    grads = np.zeros(total)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        a = acts[l]
        nz, ny, nx, _ = a.shape
        ap = np.pad(a, ((1, 1), (1, 1), (1, 1), (0, 0)))
        dW = np.zeros_like(W)
        for dz in range(3):
            for dy in range(3):
                for dx in range(3):
                    sub = ap[dz:dz + nz, dy:dy + ny, dx:dx + nx, :].reshape(-1, W.shape[3])
                    dW[dz, dy, dx] = sub.T @ g.reshape(-1, W.shape[4])
        w0, b0 = sl[l]
        grads[w0:b0] = dW.ravel()
        grads[b0:b0 + W.shape[4]] = g.reshape(-1, W.shape[4]).sum(axis=0)
        if l == 0:
            break
        gp = np.zeros((nz + 2, ny + 2, nx + 2, W.shape[3]))
        for dz in range(3):
            for dy in range(3):
                for dx in range(3):
                    gp[dz:dz + nz, dy:dy + ny, dx:dx + nx, :] += g @ W[dz, dy, dx].T
        g = gp[1:-1, 1:-1, 1:-1, :] * (a > 0)
    return loss, grads


def subspace_channels(x: np.ndarray, S: np.ndarray, scale: float) -> np.ndarray:
    """x: (nx, ny, nz, nq) image; returns (nz, ny, nx, 2r) channels of scale * (x S)."""
    c = np.tensordot(x, S, axes=([3], [0])) * scale          # (nx, ny, nz, r)
    c = np.transpose(c, (2, 1, 0, 3))
    return np.stack([c.real, c.imag], axis=-1).reshape(c.shape[:3] + (2 * S.shape[1],))


def subspace_image(chan: np.ndarray, S: np.ndarray, scale: float) -> np.ndarray:
    """Inverse of subspace_channels through S^H: returns the (nx, ny, nz, nq) image."""
    r = S.shape[1]
    c = chan.reshape(chan.shape[:3] + (r, 2))
    c = (c[..., 0] + 1j * c[..., 1]) / scale                  # (nz, ny, nx, r)
    c = np.transpose(c, (2, 1, 0, 3))
    return np.tensordot(c, S.conj().T, axes=([3], [0]))
