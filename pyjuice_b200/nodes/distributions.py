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
