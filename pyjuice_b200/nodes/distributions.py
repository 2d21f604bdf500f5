"""Input distributions.

Categorical, SoftEvidenceCategorical, Bernoulli, Gaussian and DiscreteLogistic. Their
parameter layouts, metadata and initialisation follow the reference's classes of the same
names (src/pyjuice/nodes/distributions/categorical.py:12-74, softevi_categorical.py,
bernoulli.py, gaussian.py, discrete_logistic.py). The forward, flow, EM and sampling
arithmetic is implemented by the CUDA kernels in ``csrc/input_kernels.cu`` (Categorical),
``csrc/input_poe.cu`` (SoftEvidenceCategorical) and ``csrc/input_dists.cu``.
"""

from __future__ import annotations

import math
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


class SoftEvidenceCategorical(Categorical):
    """Categorical distribution over ``num_cats`` categories that is multiplied, per sample, by
    external evidence over the categories (a product of experts): the node's value is
    ``log theta[x] + L[x] - log sum_k theta[k] exp(L[k])`` for log-weights L given to the
    circuit's forward and backward passes as ``categorical_evidence_logp``
    ``[B, num_vars, K]`` (optionally sparse, with ``soft_evidence_cat_ids``). Parameters,
    flows and EM are those of the Categorical
    (src/pyjuice/nodes/distributions/softevi_categorical.py:225-859)."""

    def get_signature(self):
        return "ExternSoftEvidenceCategorical"

    def requires_external_inputs(self):
        return True

    def _get_constructor(self):
        return SoftEvidenceCategorical, {"num_cats": self.num_cats}


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


class DiscreteLogistic(Distribution):
    """Discretised logistic distribution over ``num_cats`` equal bins of ``val_range``:
    parameters (mu, s) per node (location and logistic scale); bin x covers
    ``[lo + x w, lo + (x + 1) w)`` with ``w = (hi - lo) / num_cats``, the first and last bins
    reach to -inf and +inf. Three flow slots per node (flow-weighted bin midpoint, its
    square, and the flow); EM moment-matches with the standard deviation kept at or above
    ``min_std`` (src/pyjuice/nodes/distributions/discrete_logistic.py:12-202). The data are
    bin indices (any numeric dtype)."""

    def __init__(self, val_range, num_cats: int, min_std: float = 0.01, input_type: str = "discrete"):
        if input_type != "discrete":
            raise ValueError("only discrete inputs (bin indices) are supported")
        self.val_range = (float(val_range[0]), float(val_range[1]))
        self.num_cats = int(num_cats)
        self.min_std = float(min_std)
        self.input_type = input_type

    def get_signature(self):
        return "DiscreteLogistic"

    def get_metadata(self):
        return [self.val_range[0], self.val_range[1], self.num_cats, self.min_std]

    def num_parameters(self):
        return 2

    def num_param_flows(self):
        return 3

    def init_parameters(self, num_nodes: int, perturbation: float = 2.0, params: Optional[torch.Tensor] = None, **kwargs):
        """Locations ~ N(mu, std), scales std * sqrt(3) / pi shrunk by a random factor in
        (exp(-0.04 perturbation), 1]; mu defaults to the middle of the range and std to a
        quarter of its width (discrete_logistic.py:62-78)."""
        if params is not None:
            if params.numel() != num_nodes * 2:
                raise ValueError("parameter tensor has the wrong size")
            return params.contiguous()
        lo, hi = self.val_range
        mu = kwargs.get("mu", (lo + hi) / 2.0)
        std = kwargs.get("std", (hi - lo) / 4.0)
        mus = torch.normal(mean=torch.ones([num_nodes]) * mu, std=std)
        ss = torch.exp(torch.rand([num_nodes]) * -0.04 * perturbation) * std * math.sqrt(3) / math.pi
        return torch.stack((mus, ss), dim=1).reshape(-1).contiguous()

    def get_data_dtype(self):
        return torch.float32

    def _get_constructor(self):
        return DiscreteLogistic, {"val_range": self.val_range, "num_cats": self.num_cats, "min_std": self.min_std}
