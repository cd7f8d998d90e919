"""Cell partitions and the shared-node exchange of the residual across ranks.

The reference distributes the mesh with DMPlexDistribute (libsrc/pylith/topology/
Distributor.cc:127-145, overlap 0) and sums the contributions of cells on different ranks to
their shared vertices in DMLocalToGlobal(ADD_VALUES) over a PetscSF
(libsrc/pylith/topology/Field.cc:394-402, called from TimeDependent.cc:667). Here:

  * `partition_mesh` splits the cells into contiguous ranges of the locality order (the mesh is
    Morton-ordered, so each range is a compact subdomain) and gives every part its own local
    node numbering, the local-to-global node map, and, per neighbouring part, the list of
    shared local nodes sorted by global node id (so both sides agree on the order);
  * `HaloExchange.sum_shared` adds the neighbours' partial sums into the local residual at the
    shared nodes: one packed send and one receive per neighbour over torch.distributed (NCCL on
    the GPU, gloo on CPU), then one index_add. After it every rank holds, for each of its nodes,
    the same value the global residual has there.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List

import numpy as np

from .meshing import Mesh


@dataclass
class LocalMesh:
    part: int
    mesh: Mesh                       # local numbering
    cell_ids: np.ndarray             # global cell id of each local cell
    node_ids: np.ndarray             # global node id of each local node
    shared: Dict[int, np.ndarray] = field(default_factory=dict)  # part -> local node indices


def partition_mesh(mesh: Mesh, nparts: int) -> List[LocalMesh]:
    """Contiguous cell ranges of the mesh order; cohesive cells are not supported here."""
    if mesh.cohesive is not None:
        raise ValueError("partition_mesh handles domain cells only")
    nc = mesh.num_cells
    bounds = np.linspace(0, nc, nparts + 1).astype(np.int64)
    parts = []
    owner_sets = []
    for p in range(nparts):
        cells = mesh.cells[bounds[p]:bounds[p + 1]]
        nodes = np.unique(cells)
        parts.append((np.arange(bounds[p], bounds[p + 1]), nodes, cells))
        owner_sets.append(nodes)
    # node -> parts touching it
    counts = np.zeros(mesh.num_nodes, dtype=np.int64)
    for nodes in owner_sets:
        counts[nodes] += 1
    out = []
    for p, (cell_ids, nodes, cells) in enumerate(parts):
        g2l = np.full(mesh.num_nodes, -1, dtype=np.int64)
        g2l[nodes] = np.arange(len(nodes))
        local = Mesh(mesh.cell_type, np.ascontiguousarray(mesh.coords[nodes]),
                     g2l[cells].astype(np.int32))
        lm = LocalMesh(p, local, cell_ids, nodes)
        multi = nodes[counts[nodes] > 1]
        for q in range(nparts):
            if q == p:
                continue
            common = np.intersect1d(multi, owner_sets[q], assume_unique=True)
            if len(common):
                lm.shared[q] = g2l[common]  # sorted by global id
        out.append(lm)
    return out


class HaloExchange:
    """Sum of partial nodal values across the parts that share nodes (ADD_VALUES)."""

    def __init__(self, local: LocalMesh, device=None, group=None):
        import torch

        self.local = local
        self.group = group
        self.device = device if device is not None else torch.device("cpu")
        self.peers = sorted(local.shared)
        self.index = {q: torch.as_tensor(local.shared[q], dtype=torch.int64, device=self.device)
                      for q in self.peers}

    def sum_shared(self, r) -> None:
        """r: tensor [3 * num_local_nodes] (any float dtype), updated in place."""
        import torch
        import torch.distributed as dist

        r3 = r.view(-1, 3)
        sends = {q: r3.index_select(0, self.index[q]).contiguous() for q in self.peers}
        recvs = {q: torch.empty_like(sends[q]) for q in self.peers}
        ops = []
        for q in self.peers:
            ops.append(dist.P2POp(dist.isend, sends[q], q, group=self.group))
            ops.append(dist.P2POp(dist.irecv, recvs[q], q, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for q in self.peers:
            r3.index_add_(0, self.index[q], recvs[q])
