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
    shared nodes: one pack kernel, one send and one receive per neighbour over torch.distributed
    (NCCL on the GPU, gloo on CPU), then one add kernel. After it every rank holds, for each of
    its nodes, the same value the global residual has there.
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
    """Sum of partial nodal values across the parts that share nodes (ADD_VALUES).

    On CUDA tensors the shared nodes' values are packed into one send buffer and the neighbours'
    values added back by the library's kernels (pl_halo_pack / pl_halo_unpack_add, one launch
    each, on the context's stream); between them each neighbour's slice moves by point-to-point
    send/receive (NCCL). On CPU tensors (the gloo transport of the multi-process CPU tests) the
    same two steps are index_select and index_add.
    """

    def __init__(self, local: LocalMesh, device=None, group=None, ctx=None):
        import torch

        self.local = local
        self.group = group
        self.device = torch.device(device) if device is not None else torch.device("cpu")
        self.peers = sorted(local.shared)
        self.counts = [len(local.shared[q]) for q in self.peers]
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        self.total = int(self.offsets[-1])
        nodes = (np.concatenate([local.shared[q] for q in self.peers]) if self.peers
                 else np.zeros(0, dtype=np.int64))
        self.halo = None
        if self.device.type == "cuda":
            import ctypes

            from . import _lib as C

            if ctx is None:
                raise ValueError("a CUDA exchange needs the pylith_b200 Context of its device")
            self.ctx = ctx
            counts = np.ascontiguousarray(self.counts, dtype=np.int64)
            nodes32 = np.ascontiguousarray(nodes, dtype=np.int32)
            h = ctypes.c_void_p()
            C.check(C.lib().pl_halo_create(ctx.handle, len(self.peers), counts.ctypes.data,
                                           nodes32.ctypes.data, ctypes.byref(h)))
            self.halo = h
        else:
            self.index = torch.as_tensor(nodes, dtype=torch.int64)

    def close(self):
        if self.halo:
            from . import _lib as C

            C.lib().pl_halo_destroy(self.halo)
            self.halo = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def slices(self, buf):
        """{neighbour: its part of a send or receive buffer}."""
        return {q: buf[3 * self.offsets[i]:3 * self.offsets[i + 1]] for i, q in enumerate(self.peers)}

    def pack(self, r, out=None):
        """The shared nodes' values of r, neighbour after neighbour: [3 * entries]."""
        import torch

        if out is None:
            out = torch.empty(3 * self.total, dtype=r.dtype, device=r.device)
        if self.halo is not None:
            from . import _lib as C

            fn = C.lib().pl_halo_pack if r.dtype == torch.float64 else C.lib().pl_halo_pack_f32
            C.check(fn(self.halo, r.data_ptr(), out.data_ptr()))
        else:
            out.view(-1, 3).copy_(r.view(-1, 3).index_select(0, self.index))
        return out

    def unpack_add(self, recv, r) -> None:
        """Adds the neighbours' values (laid out as `pack`'s output) into r at the shared nodes."""
        import torch

        if self.halo is not None:
            from . import _lib as C

            fn = C.lib().pl_halo_unpack_add if r.dtype == torch.float64 else C.lib().pl_halo_unpack_add_f32
            C.check(fn(self.halo, recv.data_ptr(), r.data_ptr()))
        else:
            r.view(-1, 3).index_add_(0, self.index, recv.view(-1, 3))

    def sum_shared(self, r, send=None, recv=None) -> None:
        """r: tensor [3 * num_local_nodes], updated in place; send/recv: optional buffers of
        3 * entries values reused between calls."""
        import torch
        import torch.distributed as dist

        send = self.pack(r, send)
        if recv is None:
            recv = torch.empty_like(send)
        ss, rs = self.slices(send), self.slices(recv)
        ops = []
        for q in self.peers:
            ops.append(dist.P2POp(dist.isend, ss[q], q, group=self.group))
            ops.append(dist.P2POp(dist.irecv, rs[q], q, group=self.group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        self.unpack_add(recv, r)
