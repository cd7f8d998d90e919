"""Multi-rank residual assembly on CPU with the gloo backend (world size 2 and 3): each rank
computes the residual of its cell partition (oracle cell loop), the shared-node exchange adds
the neighbours' partial sums, and every rank's values equal the global residual at its nodes
(the reference's DMLocalToGlobal ADD_VALUES, libsrc/pylith/topology/Field.cc:394-402)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, result_q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import datetime

    import torch
    import torch.distributed as dist

    import oracle as O
    from pylith_b200 import materials as MAT
    from pylith_b200 import meshing as M
    from pylith_b200.parallel import HaloExchange, partition_mesh

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mesh = M.box_tet_delaunay(5000, seed=2)
        rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=1)
        u = np.random.default_rng(3).standard_normal(mesh.num_nodes * 3)
        parts = partition_mesh(mesh, world)
        lm = parts[rank]
        ids = lm.cell_ids
        aux = O.AuxFields([(rho[ids, None], "cell"), (mu[ids, None], "cell"), (K[ids, None], "cell")])
        u_loc = u.reshape(-1, 3)[lm.node_ids].ravel()
        r_loc = torch.from_numpy(O.residual(lm.mesh, u_loc, aux,
                                            f1="IsotropicLinearElasticity3D::f1v_infinitesimalStrain"))
        HaloExchange(lm).sum_shared(r_loc)
        aux_g = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
        r_glob = O.residual(mesh, u, aux_g, f1="IsotropicLinearElasticity3D::f1v_infinitesimalStrain")
        want = r_glob.reshape(-1, 3)[lm.node_ids].ravel()
        err = np.abs(r_loc.numpy() - want).max() / np.abs(want).max()
        result_q.put((rank, float(err), len(lm.shared)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_residual_matches_global(oracle_lib, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err, npeers in results:
        assert err <= 1e-13, (rank, err)
        assert npeers >= 1
