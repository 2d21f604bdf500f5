"""pyjuice_b200: PyJuice's compiled-circuit hot path on hand-written sm_100a kernels.

Same public API as the reference package for the circuit passes:
``compile`` / ``TensorCircuit``, ``inputs`` / ``multiply`` / ``summate`` /
``set_block_size``, ``distributions.Categorical``, ``structures.HCLT``,
``queries.sample`` / ``marginal`` / ``conditional``, and ``autograd.circuit_ll`` (a
differentiable soft-evidence log-likelihood).
"""

from . import nodes, layer, model, structures, queries, autograd, io
from .nodes import inputs, multiply, summate, set_block_size, distributions
from .model import TensorCircuit, compile
from .layer import InputLayer, ProdLayer, SumLayer
from .io import load, save

__all__ = ["compile", "TensorCircuit", "inputs", "multiply", "summate", "set_block_size", "distributions",
           "structures", "queries", "autograd", "io", "load", "save", "InputLayer", "ProdLayer", "SumLayer"]
