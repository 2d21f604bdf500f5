"""Saving and loading circuits in the reference's ``.jpc`` format (src/pyjuice/io/io.py:13-48,
io/serialization.py:11-103), so that files move between the two packages in both directions.

A ``.jpc`` file is a pickled list with one dict per node vector, children before parents:
``type`` ("Input" / "Product" / "Sum"), ``num_node_blocks``, ``block_size``, ``chs`` (indices
of the children in the list), ``edge_ids`` (numpy), ``params`` / ``zero_param_mask`` (numpy,
when set), for inputs ``scope`` (list of variables) and ``dist`` (the distribution object,
itself pickled), and ``source_node`` (index of the tied source). The last entry is the
root. The file format is the interface, so the field names and the nesting are the
reference's.

The distribution is pickled under the reference's class path (e.g.
``pyjuice.nodes.distributions.categorical.Categorical``) with the reference's attributes,
written opcode by opcode so that no ``pyjuice`` module has to be importable when saving;
when loading, that class path (and ours) maps to this package's class of the same name.
Categorical, Bernoulli, Gaussian, DiscreteLogistic and SoftEvidenceCategorical are covered.
"""

from __future__ import annotations

import io
import pickle
from typing import Sequence, Union

import numpy as np
import torch

from .model import TensorCircuit
from .nodes import CircuitNodes, inputs, multiply, summate
from .nodes.distributions import Bernoulli, Categorical, DiscreteLogistic, Gaussian, SoftEvidenceCategorical

_REF_MODULE = "pyjuice.nodes.distributions"
# our class -> the reference's module (under pyjuice.nodes.distributions) and class name
_REF_CLASS = {SoftEvidenceCategorical: ("softevi_categorical", "SoftEvidenceCategorical"),
              Categorical: ("categorical", "Categorical"), Bernoulli: ("bernoulli", "Bernoulli"),
              Gaussian: ("gaussian", "Gaussian"), DiscreteLogistic: ("discrete_logistic", "DiscreteLogistic")}
_OUR_CLASS = {name: cls for cls, (_, name) in _REF_CLASS.items()}


def _ref_state(dist) -> dict:
    """The instance dictionary of the reference's object of this distribution."""
    state = {"post_fw_fns": [], "post_bp_fns": [], "sampling_fns": []}
    if isinstance(dist, Categorical):
        state["num_cats"] = int(dist.num_cats)
    elif isinstance(dist, Gaussian):
        state.update(mu=dist.mu, sigma=dist.sigma, min_sigma=dist.min_sigma)
    elif isinstance(dist, DiscreteLogistic):
        state.update(val_range=tuple(dist.val_range), num_cats=int(dist.num_cats), min_std=dist.min_std,
                     input_type=dist.input_type)
    return state


def _pickle_dist(dist) -> bytes:
    """The distribution as the reference pickles it: protocol 2, GLOBAL of the reference's
    class, then either NEWOBJ and BUILD with the instance dictionary the reference's object
    carries, or (SoftEvidenceCategorical, whose reference class reduces to its constructor
    call) REDUCE on ``(num_cats,)``."""
    ref = next((v for cls, v in _REF_CLASS.items() if type(dist) is cls), None)
    if ref is None:
        raise NotImplementedError(f"saving distribution {type(dist).__name__} is not supported")
    out = io.BytesIO()
    out.write(b"\x80\x02")                                                    # PROTO 2
    out.write(b"c" + f"{_REF_MODULE}.{ref[0]}".encode() + b"\n" + ref[1].encode() + b"\n")  # GLOBAL
    if isinstance(dist, SoftEvidenceCategorical):
        out.write(pickle.dumps((int(dist.num_cats),), protocol=2)[2:-1])      # the argument tuple
        out.write(b"R.")                                                      # REDUCE, STOP
        return out.getvalue()
    out.write(b")\x81")                                                       # EMPTY_TUPLE, NEWOBJ
    out.write(pickle.dumps(_ref_state(dist), protocol=2)[2:-1])               # the dict (no PROTO / STOP)
    out.write(b"b.")                                                          # BUILD, STOP
    return out.getvalue()


class _DistUnpickler(pickle.Unpickler):
    def find_class(self, module, name):
        if name in _OUR_CLASS and (module.startswith(_REF_MODULE) or
                                   module.startswith("pyjuice_b200.nodes.distributions")):
            return _OUR_CLASS[name]
        raise pickle.UnpicklingError(f"distribution class {module}.{name} is not supported")


def _unpickle_dist(blob: bytes):
    dist = _DistUnpickler(io.BytesIO(blob)).load()
    for attr in ("post_fw_fns", "post_bp_fns", "sampling_fns"):
        dist.__dict__.pop(attr, None)
    if hasattr(dist, "num_cats"):
        dist.num_cats = int(dist.num_cats)
    if isinstance(dist, DiscreteLogistic):
        dist.val_range = (float(dist.val_range[0]), float(dist.val_range[1]))
    return dist


def serialize_nodes(root_ns: CircuitNodes) -> list:
    nodes_list, ns2id = [], dict()
    for ns in root_ns:
        info = {"type": "Input" if ns.is_input() else ("Product" if ns.is_prod() else "Sum"),
                "num_node_blocks": ns.num_node_blocks, "block_size": ns.block_size,
                "chs": tuple(ns2id[cs] for cs in ns.chs)}
        if ns.is_prod() or ns.is_sum():
            info["edge_ids"] = ns.edge_ids.detach().cpu().numpy().copy()
        if getattr(ns, "_params", None) is not None:
            info["params"] = ns._params.detach().cpu().numpy().copy()
        if getattr(ns, "_zero_param_mask", None) is not None:
            info["zero_param_mask"] = ns._zero_param_mask.detach().cpu().numpy().copy()
        if ns.is_input():
            info["scope"] = ns.scope.to_list()
            info["dist"] = _pickle_dist(ns.dist)
        ns2id[ns] = len(nodes_list)
        nodes_list.append(info)
    for ns in root_ns:
        if getattr(ns, "_source_node", None) is not None:
            nodes_list[ns2id[ns]]["source_node"] = ns2id[ns._source_node]
    return nodes_list


def deserialize_nodes(nodes_list: Sequence[dict]) -> CircuitNodes:
    id2ns = dict()
    for ns_id, info in enumerate(nodes_list):
        if "num_node_blocks" in info:
            nblocks, bs = info["num_node_blocks"], info["block_size"]
        elif "num_node_groups" in info:  # older files: blocks were called groups
            nblocks, bs = info["num_node_groups"], info["group_size"]
        else:
            nblocks, bs = info["num_nodes"], 1
        if info["type"] == "Input":
            ns = inputs(info["scope"], nblocks, _unpickle_dist(info["dist"]), block_size=bs)
            if "params" in info:
                ns.set_params(torch.from_numpy(np.asarray(info["params"])), normalize=False)
        elif info["type"] == "Product":
            chs = [id2ns[c] for c in info["chs"]]
            edge_ids = torch.from_numpy(np.asarray(info["edge_ids"]))
            ns = multiply(*chs, edge_ids=edge_ids, sparse_edges=edge_ids.size(0) != chs[0].num_node_blocks)
        else:
            chs = [id2ns[c] for c in info["chs"]]
            params = torch.from_numpy(np.asarray(info["params"])) if "params" in info else None
            ns = summate(*chs, edge_ids=torch.from_numpy(np.asarray(info["edge_ids"])), params=params, block_size=bs)
            if "zero_param_mask" in info:
                ns.set_zero_param_mask(torch.from_numpy(np.asarray(info["zero_param_mask"])))
        id2ns[ns_id] = ns
    for ns_id, info in enumerate(nodes_list):
        if "source_node" in info:
            id2ns[ns_id]._source_node = id2ns[info["source_node"]]
    return id2ns[len(nodes_list) - 1]


def save(fname: str, model: Union[CircuitNodes, TensorCircuit]):
    """Save an uncompiled or compiled circuit to ``fname`` (".jpc"); a compiled circuit's
    current parameters are written back to its nodes first (``update_parameters``)."""
    if isinstance(model, TensorCircuit):
        model.update_parameters()
        root_ns = model.root_ns
    else:
        root_ns = model
    if not fname.endswith(".jpc"):
        raise ValueError(f"Unknown file type `.{fname.split('.')[-1]}`.")
    with open(fname, "wb") as f:
        pickle.dump(serialize_nodes(root_ns), f)


def load(fname: str) -> CircuitNodes:
    """Load a circuit (its root node vector) from a ".jpc" file."""
    if not fname.endswith(".jpc"):
        raise ValueError(f"Unknown file type `.{fname.split('.')[-1]}`.")
    with open(fname, "rb") as f:
        nodes_list = pickle.load(f)
    return deserialize_nodes(nodes_list)
