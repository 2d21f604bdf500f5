"""Seeded synthetic datasets that stand in for the reference's benchmark data.

The reference benchmarks on MNIST-like 28x28 images with 256 grey levels; no dataset
is available here, so these generators produce data of the same shapes and value
ranges:

* ``tree_bayes_net_data``: samples of a random tree-structured Bayesian network over
  categorical variables (random spanning tree, root marginal and CPT rows drawn from
  Dirichlet(alpha)), drawn ancestrally;
* ``gaussian_field_data``: images of Gaussian random fields (white noise filtered in
  Fourier space with ``exp(-2 pi^2 l^2 |k|^2)``, length scale ``l`` pixels),
  standardised and quantised to ``num_cats`` levels through the normal CDF.
"""

from __future__ import annotations

import numpy as np
import torch


def tree_bayes_net_data(num_vars: int = 64, num_cats: int = 4, num_samples: int = 8192, alpha: float = 0.5,
                        seed: int = 0) -> torch.Tensor:
    rng = np.random.Generator(np.random.PCG64(seed))
    parent = np.full(num_vars, -1, dtype=np.int64)
    for v in range(1, num_vars):
        parent[v] = rng.integers(0, v)
    perm = rng.permutation(num_vars)          # relabel the variables
    root_p = rng.dirichlet(np.full(num_cats, alpha))
    cpts = rng.dirichlet(np.full(num_cats, alpha), size=(num_vars, num_cats))  # [v, parent value, value]
    x = np.zeros([num_samples, num_vars], dtype=np.int64)
    u = rng.random([num_samples, num_vars])
    for v in range(num_vars):                 # parents precede children in the unpermuted order
        if parent[v] < 0:
            probs = np.broadcast_to(root_p, (num_samples, num_cats))
        else:
            probs = cpts[v][x[:, parent[v]]]
        cdf = np.cumsum(probs, axis=1)
        x[:, v] = np.minimum((u[:, v:v + 1] > cdf).sum(axis=1), num_cats - 1)
    out = np.zeros_like(x)
    out[:, perm] = x
    return torch.from_numpy(out)


def gaussian_field_data(num_samples: int, side: int = 28, num_cats: int = 256, length_scale: float = 3.0,
                        channels: int = 1, seed: int = 0, chunk: int = 4096) -> torch.Tensor:
    """``[num_samples, channels * side * side]`` int64 values in ``[0, num_cats)``."""
    gen = torch.Generator().manual_seed(seed)
    fy = torch.fft.fftfreq(side)
    fx = torch.fft.rfftfreq(side)
    k2 = fy[:, None] ** 2 + fx[None, :] ** 2
    filt = torch.exp(-2.0 * (np.pi ** 2) * (length_scale ** 2) * k2)
    out = torch.empty([num_samples, channels * side * side], dtype=torch.long)
    for s in range(0, num_samples, chunk):
        e = min(s + chunk, num_samples)
        noise = torch.randn([e - s, channels, side, side], generator=gen, dtype=torch.float64)
        field = torch.fft.irfft2(torch.fft.rfft2(noise) * filt, s=(side, side))
        field = (field - field.mean(dim=(2, 3), keepdim=True)) / (field.std(dim=(2, 3), keepdim=True) + 1e-12)
        q = torch.floor(num_cats * torch.special.ndtr(field)).clamp(0, num_cats - 1).long()
        out[s:e] = q.reshape(e - s, -1)
    return out
