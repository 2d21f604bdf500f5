"""Helpers over circuit DAGs."""

from __future__ import annotations

from functools import reduce
from typing import Sequence, Union

from .nodes import CircuitNodes
from .scope import BitSet


def get_subsumed_scopes(root_ns, scopes: Union[Sequence[BitSet], Sequence[int], BitSet], type: str = "any"):
    """Every distinct node scope of the circuit that contains one of ``scopes`` ("any") or
    that meets their union ("all"), as in src/pyjuice/nodes/methods/scope.py:10-45. The result
    feeds ``TensorCircuit.enable_partial_evaluation``."""
    if not isinstance(root_ns, CircuitNodes):
        root_ns = root_ns.root_ns
    if isinstance(scopes, BitSet):
        scopes = [scopes]
    scopes = [BitSet.from_array([s]) if isinstance(s, int) else s for s in scopes]
    found, out = set(), []
    if type == "any":
        test = lambda sc: any(sc.contains_all(r) for r in scopes)
    elif type == "all":
        ref = reduce(lambda a, b: a | b, scopes)
        test = lambda sc: sc.contains_any(ref)
    else:
        raise ValueError("type must be 'any' or 'all'")
    for ns in root_ns:
        if ns.scope not in found and test(ns.scope):
            found.add(ns.scope)
            out.append(ns.scope)
    return out
