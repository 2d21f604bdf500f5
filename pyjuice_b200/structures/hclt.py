"""Hidden Chow-Liu Trees (HCLT).

Same construction as the reference (src/pyjuice/structures/hclt.py:67-125 and
src/pyjuice/structures/compilation.py:12-102):

1. pairwise mutual information of the variables, estimated with Gaussian soft
   binning (``mutual_information``, hclt.py:10-36);
2. maximum spanning tree of the MI graph. The reference calls networkx's Kruskal
   ``minimum_spanning_tree`` on weights ``-MI``; this module runs its own Kruskal with
   the same edge order (weights ascending, ties in lexicographic (u, v) order), keeps
   each node's neighbours in edge-insertion order, and derives the root (first
   minimum-eccentricity node), the BFS children and the DFS post-order from those
   adjacency lists, so the same MI matrix gives the same tree and the same node
   creation order without networkx;
3. every variable becomes a latent sum region over ``num_latents`` nodes whose product
   child joins the children's regions and the variable's own input nodes.
"""

from __future__ import annotations

from collections import deque
from typing import Dict, List, Optional, Sequence, Tuple, Type

import numpy as np
import torch

from ..nodes import inputs, multiply, set_block_size, summate
from ..nodes.distributions import Categorical, Distribution


def mutual_information(x1: torch.Tensor, x2: torch.Tensor, num_bins: int, sigma: float) -> torch.Tensor:
    B, K1 = x1.size()
    K2 = x2.size(1)
    x1 = (x1 - torch.min(x1)) / (torch.max(x1) - torch.min(x1) + 1e-8)
    x2 = (x2 - torch.min(x2)) / (torch.max(x2) - torch.min(x2) + 1e-8)
    bins = torch.linspace(0, 1, num_bins, device=x1.device)
    p1 = torch.exp(-0.5 * (x1.unsqueeze(2) - bins.view(1, 1, -1)).pow(2) / sigma ** 2)
    p2 = torch.exp(-0.5 * (x2.unsqueeze(2) - bins.view(1, 1, -1)).pow(2) / sigma ** 2)
    p12 = torch.einsum("bia,baj->ij", p1.reshape(B, K1 * num_bins, 1),
                       p2.reshape(B, 1, K2 * num_bins)).reshape(K1, num_bins, K2, num_bins) / B
    p1n = (p1 / p1.sum(dim=2, keepdim=True)).mean(dim=0)
    p2n = (p2 / p2.sum(dim=2, keepdim=True)).mean(dim=0)
    p12n = p12 / p12.sum(dim=(1, 3), keepdim=True)
    h1 = -(p1n * torch.log(p1n + 1e-4)).sum(dim=1)
    h2 = -(p2n * torch.log(p2n + 1e-4)).sum(dim=1)
    h12 = -(p12n * torch.log(p12n + 1e-4)).sum(dim=(1, 3))
    return h1.unsqueeze(1) + h2.unsqueeze(0) - h12


def mutual_information_chunked(x1: torch.Tensor, x2: torch.Tensor, num_bins: int, sigma: float,
                               chunk_size: int) -> torch.Tensor:
    K = x1.size(1)
    mi = torch.zeros([K, K])
    for xs in range(0, K, chunk_size):
        xe = min(xs + chunk_size, K)
        for ys in range(0, K, chunk_size):
            ye = min(ys + chunk_size, K)
            mi[xs:xe, ys:ye] = mutual_information(x1[:, xs:xe], x2[:, ys:ye], num_bins, sigma)
    return mi


class ChowLiuTree:
    """A spanning tree with neighbour lists in edge-insertion order."""

    def __init__(self, num_nodes: int, edges: List[Tuple[int, int]]):
        self.num_nodes = num_nodes
        self.edges = edges
        self.adj: Dict[int, List[int]] = {v: [] for v in range(num_nodes)}
        for u, v in edges:
            self.adj[u].append(v)
            self.adj[v].append(u)

    def center(self) -> int:
        ecc = []
        for s in range(self.num_nodes):
            dist = {s: 0}
            q = deque([s])
            while q:
                n = q.popleft()
                for m in self.adj[n]:
                    if m not in dist:
                        dist[m] = dist[n] + 1
                        q.append(m)
            ecc.append(max(dist.values()))
        r = min(ecc)
        return [v for v in range(self.num_nodes) if ecc[v] == r][0]

    def bfs_children(self, root: int) -> Dict[int, List[int]]:
        ch = {v: [] for v in range(self.num_nodes)}
        seen = {root}
        q = deque([root])
        while q:
            n = q.popleft()
            for m in self.adj[n]:
                if m not in seen:
                    seen.add(m)
                    ch[n].append(m)
                    q.append(m)
        return ch

    def dfs_postorder(self, root: int) -> List[int]:
        out = []
        seen = {root}
        stack = [(root, iter(self.adj[root]))]
        while stack:
            n, it = stack[-1]
            nxt = None
            for m in it:
                if m not in seen:
                    nxt = m
                    break
            if nxt is None:
                stack.pop()
                out.append(n)
            else:
                seen.add(nxt)
                stack.append((nxt, iter(self.adj[nxt])))
        return out


def chow_liu_tree(mi: np.ndarray) -> ChowLiuTree:
    """Maximum-MI spanning tree (Kruskal on -MI, ties broken in (u, v) order)."""
    K = mi.shape[0]
    iu, iv = np.triu_indices(K, k=1)
    w = -mi[iu, iv].astype(np.float64)
    order = np.argsort(w, kind="stable")
    parent = list(range(K))

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    edges = []
    for e in order:
        u, v = int(iu[e]), int(iv[e])
        ru, rv = find(u), find(v)
        if ru != rv:
            parent[ru] = rv
            edges.append((u, v))
            if len(edges) == K - 1:
                break
    return ChowLiuTree(K, edges)


def _max_cdf_power_of_2(val: int) -> int:
    count = 0
    while val % 2 == 0 and val > 0:
        val //= 2
        count += 1
    return 2 ** count


def hclt_from_tree(node_seq: Sequence[int], children: Dict[int, Sequence[int]], root: int, num_latents: int,
                   input_dist: Optional[Distribution] = None, num_root_ns: int = 1,
                   block_size: Optional[int] = None, tie_input_params: bool = False,
                   sum_edge_ids_constructor=None):
    """Build the HCLT circuit of a rooted tree (structures/compilation.py:12-102).

    ``node_seq`` is the post-order in which variables are turned into regions and
    ``children[v]`` the ordered children of ``v``.
    """
    if input_dist is None:
        input_dist = Categorical(num_cats=256)
    dist_cls, dist_kwargs = input_dist._get_constructor()
    if block_size is None:
        block_size = min(1024, _max_cdf_power_of_2(num_latents))
    num_node_blocks = num_latents // block_size
    template = None

    def leaf(v):
        nonlocal template
        if tie_input_params:
            if template is None:
                template = inputs(v, num_node_blocks=num_node_blocks, dist=dist_cls(**dist_kwargs))
                return template
            return template.duplicate(v, tie_params=True)
        return inputs(v, num_node_blocks=num_node_blocks, dist=dist_cls(**dist_kwargs))

    var2r = dict()
    with set_block_size(block_size):
        for v in node_seq:
            chs = list(children.get(v, []))
            if len(chs) == 0:
                var2r[v] = leaf(v)
            else:
                regions = [var2r[c] for c in chs]
                regions.append(leaf(v))
                rp = multiply(*regions)
                if v == root:
                    if num_root_ns == 1:
                        r = summate(rp, num_node_blocks=1, block_size=1,
                                    sum_edge_ids_constructor=sum_edge_ids_constructor)
                    else:
                        r = summate(rp, num_node_blocks=num_root_ns // block_size, block_size=block_size,
                                    sum_edge_ids_constructor=sum_edge_ids_constructor)
                else:
                    r = summate(rp, num_node_blocks=num_node_blocks, sum_edge_ids_constructor=sum_edge_ids_constructor)
                var2r[v] = r
    return var2r[root]


def HCLT(x: torch.Tensor, num_latents: int, num_bins: int = 32, sigma: float = 0.5 / 32, chunk_size: int = 64,
         num_root_ns: int = 1, block_size: Optional[int] = None, input_dist: Optional[Distribution] = None,
         input_node_type: Type[Distribution] = Categorical, input_node_params: dict = {"num_cats": 256},
         tie_input_params: bool = False, sum_edge_ids_constructor=None):
    """Hidden Chow-Liu Tree over the columns of ``x`` ([num_samples, num_vars])."""
    if input_dist is None:
        input_dist = input_node_type(**input_node_params)
    mi = mutual_information_chunked(x, x, num_bins, sigma, chunk_size=chunk_size).detach().cpu().numpy()
    tree = chow_liu_tree(mi)
    root = tree.center()
    return hclt_from_tree(tree.dfs_postorder(root), tree.bfs_children(root), root, num_latents,
                          input_dist=input_dist, num_root_ns=num_root_ns, block_size=block_size,
                          tie_input_params=tie_input_params, sum_edge_ids_constructor=sum_edge_ids_constructor)
