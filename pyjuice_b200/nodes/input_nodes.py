"""Input node vectors (reference: src/pyjuice/nodes/input_nodes.py:13)."""

from __future__ import annotations

from copy import deepcopy
from typing import Optional, Sequence, Union

import torch

from .distributions import Distribution
from .nodes import CircuitNodes
from .scope import BitSet


class InputNodes(CircuitNodes):
    def __init__(self, num_node_blocks: int, scope: Union[Sequence[int], BitSet], dist: Distribution,
                 params: Optional[torch.Tensor] = None, block_size: int = 0, **kwargs):
        if not isinstance(scope, BitSet):
            scope = BitSet.from_array(scope)
        super().__init__(num_node_blocks, scope, block_size=block_size, **kwargs)
        self.chs = []
        self.dist = dist
        self._param_initialized = False
        if params is not None:
            self.set_params(params)

    def is_input(self):
        return True

    @property
    def num_edges(self):
        return 0

    def has_params(self):
        if self.is_tied():
            return self.get_source_ns().has_params()
        return self._param_initialized and self._params is not None

    def duplicate(self, scope=None, tie_params: bool = False) -> "InputNodes":
        if scope is None:
            scope = self.scope
        elif isinstance(scope, int):
            scope = [scope]
        ns = InputNodes(self.num_node_blocks, scope=scope, dist=deepcopy(self.dist), block_size=self.block_size,
                        source_node=self if tie_params else None)
        if self.provided("_params") and not tie_params:
            ns._params = self._params.clone()
            ns._param_initialized = True
        return ns

    def get_params(self):
        return self._params

    def set_params(self, params: torch.Tensor, normalize: bool = True):
        if params.numel() != self.num_nodes * self.dist.num_parameters():
            raise ValueError("parameter tensor has the wrong number of elements")
        params = params.reshape(-1).float()
        if normalize:
            params = self.dist.normalize_parameters(params)
        self._params = params
        self._param_initialized = True

    def init_parameters(self, perturbation: float = 2.0, recursive: bool = True, is_root: bool = True,
                        ret_params: bool = False, **kwargs):
        if not self.is_tied() and not self.has_params():
            self._params = self.dist.init_parameters(num_nodes=self.num_nodes, perturbation=perturbation)
            self._param_initialized = True
            if ret_params:
                return self._params
        elif ret_params:
            return self.get_source_ns()._params

    def get_data_dtype(self):
        return self.dist.get_data_dtype()

    def __repr__(self):
        return f"InputNodes(num_node_blocks={self.num_node_blocks}, block_size={self.block_size}, dist={type(self.dist).__name__})"
