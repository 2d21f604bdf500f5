"""Circuit node vectors: the DAG the compiler turns into layers.

Mirrors the reference's ``CircuitNodes`` (src/pyjuice/nodes/nodes.py:65): a node
vector holds ``num_node_blocks`` blocks of ``block_size`` nodes that share children
and scope. Iteration order is the reference's: DFS post-order over ``chs`` (children
before parents, each vector once), or a Kahn-style top-down order when ``reverse``
is requested (nodes.py:13-62). The compiler, the parameter-update tables and the
parameter initialisation all depend on this order.
"""

from __future__ import annotations

from collections import deque
from typing import Callable, Optional

from .scope import BitSet


def node_iterator(root_ns: "CircuitNodes", reverse: bool = False):
    if not reverse:
        visited = set()
        order = []
        stack = [(root_ns, 0)]
        # Iterative post-order DFS (deep HMM chains exceed Python's recursion limit).
        while stack:
            ns, i = stack.pop()
            if i == 0:
                if ns in visited:
                    continue
                visited.add(ns)
            if i < len(ns.chs):
                stack.append((ns, i + 1))
                cs = ns.chs[i]
                if cs not in visited:
                    stack.append((cs, 0))
            else:
                order.append(ns)
        for ns in order:
            yield ns
    else:
        parcount = dict()
        for ns in node_iterator(root_ns, reverse=False):
            for cs in ns.chs:
                parcount[cs] = parcount.get(cs, 0) + 1
        queue = deque([root_ns])
        order = []
        while queue:
            ns = queue.popleft()
            order.append(ns)
            for cs in ns.chs:
                parcount[cs] -= 1
                if parcount[cs] == 0:
                    queue.append(cs)
        for ns in order:
            yield ns


class CircuitNodes:
    """Base class of input, product and sum node vectors."""

    DEFAULT_BLOCK_SIZE = 1

    def __init__(self, num_node_blocks: int, scope: BitSet, block_size: int = 0,
                 source_node: Optional["CircuitNodes"] = None, **kwargs):
        if block_size == 0:
            block_size = CircuitNodes.DEFAULT_BLOCK_SIZE
        if num_node_blocks <= 0:
            raise ValueError("`num_node_blocks` must be positive.")
        if block_size <= 0 or (block_size & (block_size - 1)) != 0:
            raise ValueError(f"`block_size` must be a power of 2, but got `block_size={block_size}`.")

        self.num_node_blocks = int(num_node_blocks)
        self.block_size = int(block_size)
        self._scope = scope
        self.chs = []

        self._output_ind_range = None
        self._param_ids = None
        self._params = None

        if source_node is not None:
            while source_node._source_node is not None:
                source_node = source_node._source_node
        self._source_node = source_node
        self._reverse_iter = False

    @property
    def scope(self) -> BitSet:
        return self._scope

    def is_sum(self):
        return False

    def is_prod(self):
        return False

    def is_input(self):
        return False

    @property
    def num_chs(self):
        return len(self.chs)

    @property
    def num_nodes(self):
        return self.num_node_blocks * self.block_size

    @property
    def num_vars(self):
        return len(self.scope)

    def is_tied(self):
        return self._source_node is not None

    def get_source_ns(self):
        return self._source_node if self.is_tied() else self

    def provided(self, name):
        return hasattr(self, name) and getattr(self, name) is not None

    def has_params(self):
        if not self.is_tied():
            return self.provided("_params")
        return self.get_source_ns().provided("_params")

    def init_parameters(self, perturbation: float = 2.0, recursive: bool = True, is_root: bool = True, **kwargs):
        if recursive:
            for ns in self:
                if ns is not self:
                    ns.init_parameters(perturbation=perturbation, recursive=False, is_root=False, **kwargs)

    def num_parameters(self, count_input_params: bool = False):
        count = 0
        for ns in self:
            if ns.is_sum() and not ns.is_tied():
                count += ns.num_edges
            elif ns.is_input() and count_input_params and not ns.is_tied():
                count += ns.num_nodes * ns.dist.num_parameters()
        return count

    def contains(self, ns: "CircuitNodes"):
        return any(n is ns for n in self)

    def _clear_tensor_circuit_hooks(self):
        for ns in self:
            for name in ("_param_range", "_param_ids", "_inverse_param_ids", "_param_flow_range",
                         "_param_flow_ids", "_output_ind_range"):
                if hasattr(ns, name):
                    setattr(ns, name, None)

    def __iter__(self):
        return node_iterator(self, self._reverse_iter)

    def __call__(self, reverse: bool = False):
        self._reverse_iter = reverse
        return self

    def __len__(self):
        return sum(1 for _ in node_iterator(self))
