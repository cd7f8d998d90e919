"""The partitioned residual on one GPU: the product kernels run on 2 and 3 cell partitions of one
mesh (each partition its own device mesh and integrator), the library's pack and add kernels
(pl_halo_pack / pl_halo_unpack_add) exchange the shared nodes' partial sums -- the transfers
between partitions are copies inside this process instead of NCCL sends -- and every partition
then holds the global residual and Jacobian action at its nodes: the global GPU result and the
oracle's (DMLocalToGlobal with ADD_VALUES, libsrc/pylith/topology/Field.cc:394-402).
FP64 tolerance: relative L2 <= 1e-12."""
import numpy as np
import pytest

from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M
from pylith_b200.parallel import HaloExchange, partition_mesh

pytestmark = pytest.mark.gpu

F1_ILE = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
JF3_ILE = "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def ctx():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


def exchange_in_process(halos, bufs):
    """Every partition's send buffer is packed; partition p receives, from each neighbour q, q's
    slice for p (both list their common nodes by global id); then adds them."""
    import torch

    sends = [h.pack(b) for h, b in zip(halos, bufs)]
    for p, (h, b) in enumerate(zip(halos, bufs)):
        recv = torch.empty_like(sends[p])
        rs = h.slices(recv)
        for q in h.peers:
            rs[q].copy_(halos[q].slices(sends[q])[p])
        h.unpack_add(recv, b)


@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("kind", ["tet4", "hex8"])
def test_partitioned_residual_and_action_match_global(oracle_lib, ctx, nparts, kind):
    import torch

    from pylith_b200 import feassemble as FA

    O = oracle_lib
    mesh = M.box_tet_delaunay(20000, seed=7) if kind == "tet4" else M.box_hex(12, 10, 8)
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=8)
    rng = np.random.default_rng(9)
    u = rng.standard_normal(mesh.num_dof)
    v = rng.standard_normal(mesh.num_dof)
    aux = O.AuxFields([(rho[:, None], "cell"), (mu[:, None], "cell"), (K[:, None], "cell")])
    r_orc = O.residual(mesh, u, aux, f1=F1_ILE)
    jv_orc = O.jacobian_action(mesh, v, aux, g3=JF3_ILE)
    # the whole mesh on the GPU
    ig = MAT.IsotropicLinearElasticity(rho, mu, K).create_integrator(FA.DeviceMesh(ctx, mesh))
    du, dv = torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()
    r_glob, jv_glob = torch.empty_like(du), torch.empty_like(du)
    ig.compute_lhs_residual(0.0, 0.0, du, r_glob)
    ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du, dv, jv_glob)
    # the partitions
    parts = partition_mesh(mesh, nparts)
    assert all(len(lm.shared) >= 1 for lm in parts)
    dms, igs, halos, rs, jvs = [], [], [], [], []
    for lm in parts:
        ids = lm.cell_ids
        dm = FA.DeviceMesh(ctx, lm.mesh)
        dms.append(dm)
        igl = MAT.IsotropicLinearElasticity(rho[ids], mu[ids], K[ids]).create_integrator(dm)
        igs.append(igl)
        halos.append(HaloExchange(lm, device="cuda", ctx=ctx))
        ul = torch.from_numpy(u.reshape(-1, 3)[lm.node_ids].ravel()).cuda()
        vl = torch.from_numpy(v.reshape(-1, 3)[lm.node_ids].ravel()).cuda()
        r, jv = torch.full_like(ul, np.nan), torch.full_like(ul, np.nan)
        igl.compute_lhs_residual(0.0, 0.0, ul, r)
        igl.compute_lhs_jacobian_action(0.0, 0.0, 0.0, ul, vl, jv)
        rs.append(r)
        jvs.append(jv)
    exchange_in_process(halos, rs)
    exchange_in_process(halos, jvs)
    ctx.synchronize()
    rg, jg = r_glob.cpu().numpy().reshape(-1, 3), jv_glob.cpu().numpy().reshape(-1, 3)
    for lm, r, jv in zip(parts, rs, jvs):
        nid = lm.node_ids
        assert rel_l2(r.cpu().numpy(), rg[nid].ravel()) <= 1e-12
        assert rel_l2(jv.cpu().numpy(), jg[nid].ravel()) <= 1e-12
        assert rel_l2(r.cpu().numpy(), r_orc.reshape(-1, 3)[nid].ravel()) <= 1e-12
        assert rel_l2(jv.cpu().numpy(), jv_orc.reshape(-1, 3)[nid].ravel()) <= 1e-12
    # the add step is deterministic: a second exchange of the same partial sums agrees bit for bit
    again = []
    for igl, lm in zip(igs, parts):
        ul = torch.from_numpy(u.reshape(-1, 3)[lm.node_ids].ravel()).cuda()
        r2 = torch.empty_like(ul)
        if kind == "tet4":  # the cell-block kernels' deterministic scatter
            igl.set_scatter(FA.SCATTER_DETERMINISTIC)
        igl.compute_lhs_residual(0.0, 0.0, ul, r2)
        again.append(r2)
    exchange_in_process(halos, again)
    twice = [a.clone() for a in again]
    for igl, lm, a in zip(igs, parts, again):
        ul = torch.from_numpy(u.reshape(-1, 3)[lm.node_ids].ravel()).cuda()
        igl.compute_lhs_residual(0.0, 0.0, ul, a)
    exchange_in_process(halos, again)
    ctx.synchronize()
    if kind == "tet4":
        for a, b in zip(again, twice):
            assert torch.equal(a, b)
    for h in halos:
        h.close()
