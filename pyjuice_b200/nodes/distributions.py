"""Input distributions.

Only the Categorical distribution is on the accelerated path. Its parameter layout
(``num_cats`` probabilities per node, node-major), metadata (``[num_cats]``) and
initialisation follow the reference's ``Categorical``
(src/pyjuice/nodes/distributions/categorical.py:12-74). The forward, flow, EM and
sampling arithmetic is implemented by the CUDA kernels in ``csrc/input_kernels.cu``.
"""

from __future__ import annotations

from typing import Optional

import torch


class Distribution:
    def get_signature(self) -> str:
        raise NotImplementedError()

    def get_metadata(self):
        return []

    def num_parameters(self) -> int:
        raise NotImplementedError()

    def num_param_flows(self) -> int:
        raise NotImplementedError()

    def normalize_parameters(self, params: torch.Tensor) -> torch.Tensor:
        return params

    def init_parameters(self, num_nodes: int, perturbation: float = 2.0, params=None, **kwargs):
        raise NotImplementedError()

    def get_data_dtype(self):
        return torch.float32

    def _get_constructor(self):
        raise NotImplementedError()


class Categorical(Distribution):
    """Categorical distribution over ``num_cats`` categories."""

    def __init__(self, num_cats: int):
        if num_cats <= 0:
            raise ValueError("`num_cats` must be positive.")
        self.num_cats = int(num_cats)

    def get_signature(self):
        return "Categorical"

    def get_metadata(self):
        return [self.num_cats]

    def num_parameters(self):
        return self.num_cats

    def num_param_flows(self):
        return self.num_cats

    def normalize_parameters(self, params: torch.Tensor) -> torch.Tensor:
        params = params.reshape(-1, self.num_cats)
        params = params / params.sum(dim=1, keepdim=True)
        return params.reshape(-1)

    def init_parameters(self, num_nodes: int, perturbation: float = 2.0, params: Optional[torch.Tensor] = None, **kwargs):
        if params is not None:
            if params.numel() != num_nodes * self.num_cats:
                raise ValueError("parameter tensor has the wrong size")
            return params
        params = torch.exp(torch.rand([num_nodes, self.num_cats]) * -perturbation)
        params /= params.sum(dim=1, keepdim=True)
        return params.reshape(-1)

    def get_data_dtype(self):
        return torch.long

    def _get_constructor(self):
        return Categorical, {"num_cats": self.num_cats}


class Bernoulli(Distribution):
    """Bernoulli distribution: one parameter per node, the probability of x > 0
    (src/pyjuice/nodes/distributions/bernoulli.py:11-102). Two flow slots per node: the flow
    of samples with x > 0, and of the others."""

    def get_signature(self):
        return "Bernoulli"

    def get_metadata(self):
        return []

    def num_parameters(self):
        return 1

    def num_param_flows(self):
        return 2

    def init_parameters(self, num_nodes: int, perturbation: float = 2.0, params: Optional[torch.Tensor] = None, **kwargs):
        if params is not None:
            if params.numel() != num_nodes:
                raise ValueError("parameter tensor has the wrong size")
            return params
        params = torch.exp(torch.rand([num_nodes, 2]) * -perturbation)
        params /= params.sum(dim=1, keepdim=True)
        return params[:, 0].contiguous()

    def get_data_dtype(self):
        return torch.bool

    def _get_constructor(self):
        return Bernoulli, {}


class Gaussian(Distribution):
    """Gaussian distribution: parameters (mu, sigma) per node, sigma kept at or above
    ``min_sigma`` by EM; three flow slots per node (flow-weighted x, x^2 and 1)
    (src/pyjuice/nodes/distributions/gaussian.py:11-170). ``mu`` and ``sigma`` set the scale of
    the random initialisation."""

    def __init__(self, mu: Optional[float] = None, sigma: Optional[float] = None, min_sigma: float = 0.01):
        self.mu = mu
        self.sigma = sigma
        self.min_sigma = min_sigma

    def get_signature(self):
        return "Gaussian"

    def get_metadata(self):
        return [self.min_sigma]

    def num_parameters(self):
        return 2

    def num_param_flows(self):
        return 3

    def init_parameters(self, num_nodes: int, perturbation: float = 2.0, params: Optional[torch.Tensor] = None, **kwargs):
        if params is not None:
            if params.numel() != num_nodes * 2:
                raise ValueError("parameter tensor has the wrong size")
            return params.contiguous()
        mu = kwargs.get("mu", self.mu)
        sigma = kwargs.get("sigma", self.sigma)
        if mu is None or sigma is None:
            raise ValueError("`mu` and `sigma` are needed to initialise Gaussian parameters")
        mus = torch.normal(mean=torch.ones([num_nodes]) * mu, std=sigma)
        sigmas = (torch.exp(torch.rand([num_nodes]) * -0.04 * perturbation) * sigma).clamp(min=self.min_sigma)
        return torch.stack((mus, sigmas), dim=1).reshape(-1).contiguous()

    def get_data_dtype(self):
        return torch.float32

    def _get_constructor(self):
        return Gaussian, {"mu": self.mu, "sigma": self.sigma, "min_sigma": self.min_sigma}
