"""GPU parity: the CUDA cell loop (called through the C ABI) against the oracle on the same
seeded meshes, fields and parameters. FP64 tolerance: relative L2 <= 1e-12 (the FP64
parity bar); FP32 Jacobian action: relative L2 <= 1e-5."""
import numpy as np
import pytest

import known_answers as KA
from pylith_b200 import materials as MAT
from pylith_b200 import meshing as M

pytestmark = pytest.mark.gpu

F1_ILE = "IsotropicLinearElasticity3D::f1v_infinitesimalStrain"
JF3_ILE = "IsotropicLinearElasticity3D::Jf3vu_infinitesimalStrain"
F1_GM = "IsotropicLinearGenMaxwell3D::f1v_infinitesimalStrain"
JF3_GM = "IsotropicLinearGenMaxwell3D::Jf3vu_infinitesimalStrain"
TOL64 = 1e-12


def rel_l2(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def ctx(torch_cuda):
    from pylith_b200 import feassemble as FA

    return FA.Context(0)


def dev(torch, a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a))
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


MESHES = {
    "tet4": lambda: M.box_tet_delaunay(6000, seed=5),
    "hex8": lambda: M.box_hex(6, 5, 4),
    "hex27": lambda: M.box_hex27(3, 3, 2),
    "tet4_unsorted": lambda: M.box_tet_delaunay(3000, seed=9, reorder=False),
}


def elastic_setup(mesh, seed=0, body_force=False):
    rho, mu, K = MAT.lognormal_elastic(mesh.num_cells, seed=seed)
    bf = np.random.default_rng(seed + 1).standard_normal((mesh.num_cells, 3)) * 1e3 if body_force else None
    return MAT.IsotropicLinearElasticity(rho, mu, K, bf)


def oracle_aux(O, mat):
    fields = [(mat.density[:, None], "cell")]
    if mat.body_force is not None:
        fields.append((mat.body_force, "cell"))
    fields += [(mat.shear_modulus[:, None], "cell"), (mat.bulk_modulus[:, None], "cell")]
    return O.AuxFields(fields)


@pytest.mark.parametrize("kind", list(MESHES))
@pytest.mark.parametrize("scatter", [0, 1, 3])
def test_elastic_residual_matches_oracle(oracle_lib, torch_cuda, ctx, kind, scatter):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES[kind]()
    mat = elastic_setup(mesh)
    u = np.random.default_rng(2).standard_normal(mesh.num_nodes * 3)
    r_ref = O.residual(mesh, u, oracle_aux(O, mat), f1=F1_ILE)
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    ig.set_scatter(scatter)
    du = dev(torch, u)
    dr = torch.full_like(du, np.nan)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    # ADD mode accumulates on top of the existing values
    ig.compute_lhs_residual(0.0, 0.0, du, dr, mode=FA.ADD)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), 2 * r_ref) <= TOL64


@pytest.mark.parametrize("kind", ["tet4", "hex8", "hex27"])
def test_body_force_residual(oracle_lib, torch_cuda, ctx, kind):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES[kind]()
    mat = elastic_setup(mesh, body_force=True)
    u = np.random.default_rng(3).standard_normal(mesh.num_nodes * 3) * 1e-3
    r_ref = O.residual(mesh, u, oracle_aux(O, mat), f0="Elasticity::g0v_bodyforce", f1=F1_ILE)
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    du = dev(torch, u)
    dr = torch.zeros_like(du)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64


@pytest.mark.parametrize("kind", ["tet4", "hex8", "hex27"])
def test_jacobian_action_and_assembly_match_oracle(oracle_lib, torch_cuda, ctx, kind):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES[kind]()
    mat = elastic_setup(mesh, seed=4)
    aux = oracle_aux(O, mat)
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3=JF3_ILE))
    v = np.random.default_rng(5).standard_normal(mesh.num_nodes * 3)
    jv_ref = J @ v
    dm = FA.DeviceMesh(ctx, mesh)
    ig = mat.create_integrator(dm)
    dv = dev(torch, v)
    djv = torch.zeros_like(dv)
    ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, None, dv, djv)
    ctx.synchronize()
    assert rel_l2(djv.cpu().numpy(), jv_ref) <= TOL64
    # FP32 action (FP32 operands and accumulation, FP64 geometry)
    dv32 = dv.float()
    djv32 = torch.zeros_like(dv32)
    ig.compute_lhs_jacobian_action_f32(0.0, 0.0, dv32, djv32)
    ctx.synchronize()
    assert rel_l2(djv32.double().cpu().numpy(), jv_ref) <= 1e-5
    # assembled block-CSR Jacobian
    A = FA.Matrix(dm)
    ig.compute_lhs_jacobian(0.0, 0.0, 0.0, None, A)
    Jg = A.to_scipy().tocsr()
    assert abs(Jg - J).max() <= TOL64 * abs(J).max()
    dy = torch.zeros_like(dv)
    A.spmv(dv, dy)
    ctx.synchronize()
    assert rel_l2(dy.cpu().numpy(), jv_ref) <= TOL64


def genmaxwell_setup(mesh, seed=0):
    rng = np.random.default_rng(seed)
    nc = mesh.num_cells
    nq = M.QUAD_POINTS[mesh.cell_type]
    rho, mu, K = MAT.lognormal_elastic(nc, seed=seed)
    tau = MAT.genmaxwell_times(rho, np.sqrt(mu / rho), [1e18, 1e19, 1e20], [0.3, 0.3, 0.3])
    ratio = np.tile([0.3, 0.3, 0.3], (nc, 1))
    visc = rng.standard_normal((nc, nq, 18)) * 1e-5
    total = rng.standard_normal((nc, nq, 6)) * 1e-5
    return MAT.IsotropicLinearGenMaxwell(rho, mu, K, tau, ratio, visc, total)


def genmaxwell_oracle_aux(O, g):
    return O.AuxFields([(g.density[:, None], "cell"), (g.shear_modulus[:, None], "cell"),
                        (g.bulk_modulus[:, None], "cell"), (g.maxwell_time, "cell"),
                        (g.shear_modulus_ratio, "cell"), (g.viscous_strain, "qp"), (g.total_strain, "qp")])


@pytest.mark.parametrize("kind", ["hex8", "tet4", "hex27"])
def test_genmaxwell_residual_jacobian_and_state_update(oracle_lib, torch_cuda, ctx, kind):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES[kind]()
    g = genmaxwell_setup(mesh)
    dt = 1.0 * MAT.YEAR
    aux = genmaxwell_oracle_aux(O, g)
    u = np.random.default_rng(7).standard_normal(mesh.num_nodes * 3) * 1e-2
    r_ref = O.residual(mesh, u, aux, f1=F1_GM, constants=[dt])
    J = O.assemble(mesh, O.jacobian_elements(mesh, aux, g3=JF3_GM, constants=[dt]))
    v = np.random.default_rng(8).standard_normal(mesh.num_nodes * 3)
    visc_ref, total_ref = O.project_qp(
        mesh, u, aux, ["IsotropicLinearGenMaxwell3D::viscousStrain_infinitesimalStrain_asVector",
                       "Elasticity3D::infinitesimalStrain_asVector"], [18, 6], constants=[dt])
    dm = FA.DeviceMesh(ctx, mesh)
    ig = g.create_integrator(dm, dt)
    du, dv = dev(torch, u), dev(torch, v)
    dr, djv = torch.zeros_like(du), torch.zeros_like(du)
    ig.compute_lhs_residual(0.0, dt, du, dr)
    ig.compute_lhs_jacobian_action(0.0, dt, 0.0, du, dv, djv)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy(), J @ v) <= TOL64
    ig.update_state_vars(0.0, dt, du)
    ctx.synchronize()
    nq = M.QUAD_POINTS[mesh.cell_type]
    visc = ig.get_aux("viscous_strain", (mesh.num_cells, nq, 18))
    total = ig.get_aux("total_strain", (mesh.num_cells, nq, 6))
    assert rel_l2(visc, visc_ref) <= TOL64
    assert rel_l2(total, total_ref) <= TOL64


def test_genmaxwell_relaxation_known_answer_on_gpu(torch_cuda, ctx):
    """The analytic relaxation of axialstrain_genmaxwell_soln.py, stepped on the GPU."""
    from pylith_b200 import feassemble as FA

    torch = torch_cuda
    mesh = M.box_hex(2, 2, 2, lo=(-4000.0, -4000.0, -8000.0), hi=(4000.0, 4000.0, 0.0))
    mu, K, lam, tau = KA.genmaxwell_params()
    nc, nq, e0 = mesh.num_cells, 8, KA.GM_E0
    g = MAT.IsotropicLinearGenMaxwell(
        np.full(nc, KA.GM_DENSITY), np.full(nc, mu), np.full(nc, K), np.tile(tau, (nc, 1)),
        np.tile(KA.GM_RATIO, (nc, 1)), np.tile([-e0 / 3, -e0 / 3, 2 * e0 / 3, 0, 0, 0] * 3, (nc, nq, 1)),
        np.tile([0, 0, e0, 0, 0, 0.0], (nc, nq, 1)))
    dm = FA.DeviceMesh(ctx, mesh)
    ig = g.create_integrator(dm, KA.GM_DT)
    X = mesh.coords
    u = np.stack([0 * X[:, 0], 0 * X[:, 1], e0 * (X[:, 2] + 8000.0)], axis=1).ravel()
    du = dev(torch, u)
    dr = torch.zeros_like(du)
    for step in range(1, KA.GM_STEPS + 1):
        ig.compute_lhs_residual(step * KA.GM_DT, KA.GM_DT, du, dr)
        ig.update_state_vars(step * KA.GM_DT, KA.GM_DT, du)
        ctx.synchronize()
        sigma = KA.stress_from_residual(X, dr.cpu().numpy(), 8000.0**3)
        np.testing.assert_allclose(np.diag(sigma), KA.genmaxwell_stress(step * KA.GM_DT), rtol=1e-10)


def fault_setup(nx=4, ny=3, nz=3):
    mesh = M.insert_fault_x(M.box_hex(nx, ny, nz))
    rng = np.random.default_rng(11)
    slip = rng.standard_normal((mesh.num_lagrange, 3))
    fault = MAT.FaultCohesiveKin(slip, ref_dir_1=(0, 0, 1), ref_dir_2=(0.5, 0, 0.5))
    return mesh, fault


def test_cohesive_residual_jacobian_action_and_assembly(oracle_lib, torch_cuda, ctx):
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh, fault = fault_setup()
    u = np.random.default_rng(12).standard_normal(mesh.num_dof)
    r_ref = O.cohesive_residual(mesh, u, fault.slip, fault.constants)
    Jc = O.cohesive_jacobian(mesh, fault.constants)
    v = np.random.default_rng(13).standard_normal(mesh.num_dof)
    dm = FA.DeviceMesh(ctx, mesh)
    ig = fault.create_integrator(dm)
    du, dv = dev(torch, u), dev(torch, v)
    dr, djv = torch.zeros_like(du), torch.zeros_like(du)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du, dv, djv)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy(), Jc @ v) <= TOL64
    A = FA.Matrix(dm)
    ig.compute_lhs_jacobian(0.0, 0.0, 0.0, None, A)
    Jg = A.to_scipy().tocsr()
    assert abs(Jg - Jc).max() <= 1e-12 * abs(Jc).max()


def test_full_fault_problem_residual(oracle_lib, torch_cuda, ctx):
    """Domain + interface integrators summed into one local vector (TimeDependent's loop over
    integrators, TimeDependent.cc:659-662)."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh, fault = fault_setup(6, 4, 3)
    mat = elastic_setup(mesh, seed=21)
    u = np.random.default_rng(14).standard_normal(mesh.num_dof)
    r_ref = np.zeros(mesh.num_dof)
    r_ref[:3 * mesh.num_nodes] = O.residual(mesh, u[:3 * mesh.num_nodes], oracle_aux(O, mat), f1=F1_ILE)
    O.cohesive_residual(mesh, u, fault.slip, fault.constants, r=r_ref)
    dm = FA.DeviceMesh(ctx, mesh)
    igs = [mat.create_integrator(dm), fault.create_integrator(dm)]
    du = dev(torch, u)
    dr = torch.zeros_like(du)
    for i, ig in enumerate(igs):
        ig.compute_lhs_residual(0.0, 0.0, du, dr, mode=FA.INSERT if i == 0 else FA.ADD)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64


def test_host_buffer_entry_point(oracle_lib, torch_cuda, ctx):
    from pylith_b200 import feassemble as FA

    O = oracle_lib
    mesh = MESHES["tet4"]()
    mat = elastic_setup(mesh)
    u = np.random.default_rng(2).standard_normal(mesh.num_nodes * 3)
    r_ref = O.residual(mesh, u, oracle_aux(O, mat), f1=F1_ILE)
    ig = mat.create_integrator(FA.DeviceMesh(ctx, mesh))
    r = np.zeros_like(u)
    ig.compute_lhs_residual_host(0.0, 0.0, u, r)
    assert rel_l2(r, r_ref) <= TOL64
    # the same call with both host buffers from pl_host_alloc
    hu, hr = ctx.host_empty(u.shape), ctx.host_empty(u.shape)
    hu[:] = u
    ig.compute_lhs_residual_host(0.0, 0.0, hu, hr)
    assert rel_l2(hr, r_ref) <= TOL64


def _page_nodes(ptr: int, nbytes: int):
    """NUMA node of every 64th page of [ptr, ptr + nbytes) (move_pages query; x86-64 / arm64)."""
    import ctypes
    import platform

    nr = {"x86_64": 279, "aarch64": 239}.get(platform.machine())
    if nr is None:
        return None
    libc = ctypes.CDLL(None, use_errno=True)
    addrs = list(range(ptr, ptr + nbytes, 64 * 4096))
    pages = (ctypes.c_void_p * len(addrs))(*addrs)
    status = (ctypes.c_int * len(addrs))()
    if libc.syscall(nr, 0, ctypes.c_ulong(len(addrs)), pages, None, status, 0) != 0:
        return None
    return list(status)


def test_numa_local_host_buffers(torch_cuda, ctx):
    """pl_host_alloc: aligned, zero-filled, page-locked (CUDA sees it as pinned host memory) and,
    where the host reports the GPU's NUMA node and lets the process use that node's memory,
    placed there; a round trip through the device returns the same bytes."""
    torch = torch_cuda
    n = 3 << 20
    a = ctx.host_empty((2, n))
    assert a.shape == (2, n) and a.dtype == np.float64
    assert a.ctypes.data % 256 == 0
    assert not a.any()
    t = torch.from_numpy(a)
    assert t.is_pinned()
    a[0] = np.arange(n, dtype=np.float64)
    a[1] = -a[0]
    d = t.to("cuda", non_blocking=True)
    back = ctx.host_empty((2, n))
    torch.from_numpy(back).copy_(d * 2.0, non_blocking=True)
    torch.cuda.synchronize()
    assert np.array_equal(back, 2.0 * a)
    node = ctx.numa_node
    allowed = ""
    with open("/proc/self/status") as f:
        for ln in f:
            if ln.startswith("Mems_allowed_list:"):
                allowed = ln.split(":", 1)[1].strip()
    mems = set()
    for part in filter(None, allowed.split(",")):
        lo, _, hi = part.partition("-")
        mems |= set(range(int(lo), int(hi or lo) + 1))
    nodes = _page_nodes(a.ctypes.data, a.nbytes)
    if node >= 0 and node in mems and len(mems) > 1 and nodes is not None:
        assert sum(x == node for x in nodes) >= 0.9 * len(nodes), (node, nodes[:16])


def test_unknown_kernel_is_rejected(torch_cuda, ctx):
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA
    import oracle as O

    mesh = MESHES["hex8"]()
    ig = FA.IntegratorDomain(FA.DeviceMesh(ctx, mesh))
    # the oracle's restated kernel has the right signature but is not a registered kernel
    foreign = O.kernel(F1_ILE, "oracle")
    with pytest.raises(_lib.PylithB200Error) as e:
        ig.set_kernels_residual([FA.ResidualKernels("displacement", FA.LHS, None, foreign)])
    assert e.value.code == -2
    with pytest.raises(_lib.PylithB200Error) as e:
        ig.compute_lhs_residual(0.0, 0.0, None, None)
    assert e.value.code == -1


def test_more_than_eight_constants_are_rejected(torch_cuda, ctx):
    """Integrator::_setKernelConstants takes any number of constants; the library holds at most 8
    (the kernels on the path use 1 or 6) and rejects more with PL_ERR_UNSUPPORTED instead of
    dropping the extra ones; the previous constants stay in place."""
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA

    torch = torch_cuda
    mesh = MESHES["hex8"]()
    mat = elastic_setup(mesh)
    ig = mat.create_integrator(FA.DeviceMesh(ctx, mesh))
    ig.set_constants([1.0] * 8)
    with pytest.raises(_lib.PylithB200Error) as e:
        ig.set_constants([1.0] * 9)
    assert e.value.code == -7
    du = torch.zeros(mesh.num_dof, dtype=torch.float64, device="cuda")
    ig.compute_lhs_residual(0.0, 0.0, du, torch.empty_like(du))
    ctx.synchronize()


def test_inverted_cell_is_reported(torch_cuda, ctx):
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA

    torch = torch_cuda
    mesh = M.box_hex(2, 2, 2)
    mesh.cells[0] = mesh.cells[0][[1, 0, 3, 2, 5, 4, 7, 6]]  # mirror cell 0 -> negative |J|
    mat = elastic_setup(mesh)
    ig = mat.create_integrator(FA.DeviceMesh(ctx, mesh))
    du = torch.zeros(mesh.num_nodes * 3, dtype=torch.float64, device="cuda")
    dr = torch.zeros_like(du)
    ig.compute_lhs_residual(0.0, 0.0, du, dr)
    with pytest.raises(_lib.PylithB200Error) as e:
        ctx.synchronize()
    assert e.value.code == -6
    ctx.synchronize()  # the flag is cleared after it is reported


def test_destroy_in_any_order(torch_cuda):
    """Context, mesh and integrator handles may be released in any order (the C layer defers a
    destroy until no dependent object is left)."""
    from pylith_b200 import feassemble as FA

    c = FA.Context(0)
    mesh = M.box_hex(2, 2, 2)
    dm = FA.DeviceMesh(c, mesh)
    ig = elastic_setup(mesh).create_integrator(dm)
    A = FA.Matrix(dm)
    c.close()
    dm.close()
    du = torch_cuda.zeros(mesh.num_nodes * 3, dtype=torch_cuda.float64, device="cuda")
    ig.compute_lhs_residual(0.0, 0.0, du, du.clone())
    A.close()
    ig.close()


@pytest.mark.parametrize("kind", ["tet4", "hex8", "hex27"])
def test_derived_fields_match_oracle(oracle_lib, torch_cuda, ctx, kind, tmp_path):
    """pl_compute_derived_field (cauchy_stress, cauchy_strain of basis order 0 at the cell
    centroids, IntegratorDomain.cc:596-630) against the oracle's centroid projection; the fields
    and the solution written through DataWriterHDF5 read back unchanged."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES[kind]()
    mat = elastic_setup(mesh, seed=31)
    u = np.random.default_rng(32).standard_normal(mesh.num_dof)
    ref_s, ref_e = O.project_centroid(
        mesh, u, oracle_aux(O, mat),
        ["IsotropicLinearElasticity3D::cauchyStress_infinitesimalStrain_asVector",
         "Elasticity3D::infinitesimalStrain_asVector"], [6, 6])
    ig = mat.create_integrator(FA.DeviceMesh(ctx, mesh))
    out = torch.zeros((mesh.num_cells, 12), dtype=torch.float64, device="cuda")
    ig.compute_derived_field(0.0, 0.0, dev(torch, u), out)
    ctx.synchronize()
    got = out.cpu().numpy()
    assert rel_l2(got[:, :6], ref_s) <= TOL64
    assert rel_l2(got[:, 6:], ref_e) <= TOL64
    from pylith_b200 import hdf5 as H5
    from pylith_b200 import output as OUT

    w = OUT.DataWriterHDF5(filename=str(tmp_path / "out.h5"))
    w.open(mesh)
    w.write_vertex_field(1.0, "displacement", u[:3 * mesh.num_nodes].reshape(-1, 3))
    w.write_cell_field(1.0, "cauchy_stress", got[:, :6])
    w.write_cell_field(1.0, "cauchy_strain", got[:, 6:])
    w.close()
    f = H5.H5File(str(tmp_path / "out.h5"))
    assert np.array_equal(f.dataset("/vertex_fields/displacement")[0], u[:3 * mesh.num_nodes].reshape(-1, 3))
    assert np.array_equal(f.dataset("/cell_fields/cauchy_stress")[0], got[:, :6])
    assert np.array_equal(f.dataset("/cell_fields/cauchy_strain")[0], got[:, 6:])
    assert f.attrs("/cell_fields/cauchy_stress")["vector_field_type"] == "tensor"


def test_derived_genmaxwell_stress(oracle_lib, torch_cuda, ctx):
    """Generalized-Maxwell stress from the stored state (cauchyStress_stateVars) on P1 tets,
    whose single quadrature point is the centroid; hexahedra are rejected (-7)."""
    from pylith_b200 import _lib
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES["tet4"]()
    g = genmaxwell_setup(mesh, seed=33)
    dt = 0.1 * MAT.YEAR
    u = np.random.default_rng(34).standard_normal(mesh.num_dof) * 1e-2
    ref_s, ref_e = O.project_centroid(
        mesh, u, genmaxwell_oracle_aux(O, g),
        ["IsotropicLinearGenMaxwell3D::cauchyStress_infinitesimalStrain_asVector",
         "Elasticity3D::infinitesimalStrain_asVector"], [6, 6], constants=[dt])
    ig = g.create_integrator(FA.DeviceMesh(ctx, mesh), dt)
    out = torch.zeros((mesh.num_cells, 12), dtype=torch.float64, device="cuda")
    ig.compute_derived_field(0.0, dt, dev(torch, u), out)
    ctx.synchronize()
    got = out.cpu().numpy()
    assert rel_l2(got[:, :6], ref_s) <= TOL64
    assert rel_l2(got[:, 6:], ref_e) <= TOL64
    hexm = MESHES["hex8"]()
    ih = genmaxwell_setup(hexm, seed=35).create_integrator(FA.DeviceMesh(ctx, hexm), dt)
    with pytest.raises(_lib.PylithB200Error) as e:
        ih.compute_derived_field(0.0, dt, dev(torch, np.zeros(hexm.num_dof)),
                                 torch.zeros((hexm.num_cells, 12), dtype=torch.float64, device="cuda"))
    assert e.value.code == -7


@pytest.mark.parametrize("kind", ["tet4", "hex8", "hex27"])
def test_two_materials_on_cell_subsets(oracle_lib, torch_cuda, ctx, kind):
    """Two materials on complementary cell subsets (one IntegratorDomain per material label,
    IntegratorDomain.cc:422-453) summed into one residual and one Jacobian action; an integrator
    over an empty subset contributes nothing."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    mesh = MESHES[kind]()
    rng = np.random.default_rng(41)
    ids = [np.flatnonzero(mesh.coords[mesh.cells].mean(axis=1)[:, 0] < 0.0),
           np.flatnonzero(mesh.coords[mesh.cells].mean(axis=1)[:, 0] >= 0.0)]
    mats = [elastic_setup(M.Mesh(mesh.cell_type, mesh.coords, mesh.cells[i]), seed=42 + k) for k, i in enumerate(ids)]
    u = rng.standard_normal(mesh.num_dof)
    v = rng.standard_normal(mesh.num_dof)
    r_ref = np.zeros(mesh.num_dof)
    jv_ref = np.zeros(mesh.num_dof)
    for i, mat in zip(ids, mats):
        sub = M.Mesh(mesh.cell_type, mesh.coords, mesh.cells[i])
        aux = oracle_aux(O, mat)
        r_ref += O.residual(sub, u, aux, f1=F1_ILE)
        J = O.assemble(sub, O.jacobian_elements(sub, aux, g3=JF3_ILE))
        jv_ref += J @ v
    dm = FA.DeviceMesh(ctx, mesh)
    igs = [mat.create_integrator(dm, i) for i, mat in zip(ids, mats)]
    empty = elastic_setup(M.Mesh(mesh.cell_type, mesh.coords, mesh.cells[:0]), seed=9).create_integrator(
        dm, np.zeros(0, dtype=np.int32))
    du, dv = dev(torch, u), dev(torch, v)
    dr = torch.full_like(du, 7.0)
    djv = torch.full_like(du, 7.0)
    for k, ig in enumerate(igs + [empty]):
        mode = FA.INSERT if k == 0 else FA.ADD
        ig.compute_lhs_residual(0.0, 0.0, du, dr, mode=mode)
        ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, du, dv, djv, mode=mode)
    ctx.synchronize()
    assert rel_l2(dr.cpu().numpy(), r_ref) <= TOL64
    assert rel_l2(djv.cpu().numpy(), jv_ref) <= TOL64
    # the empty integrator alone in INSERT mode writes zeros
    empty.compute_lhs_residual(0.0, 0.0, du, dr, mode=FA.INSERT)
    ctx.synchronize()
    assert float(dr.abs().max()) == 0.0


def test_reference_compiled_kernels_drive_the_device_path(oracle_lib, torch_cuda, ctx):
    """The reference's own pointwise kernels compiled from libsrc/pylith/fekernels/*.hh
    (oracle/_ref) are registered under their names (pl_fekernel_register) and passed to the
    integrator exactly as PyLith passes them to PetscWeakForm: the device path runs with them and
    gives what it gives with the library's own addresses, for a material and a fault."""
    from pylith_b200 import feassemble as FA

    O, torch = oracle_lib, torch_cuda
    if not O.ref_available():
        pytest.skip("reference kernels not built")
    for name in O.KERNELS:
        FA.register_fekernel(name, O.kernel(name, "ref"))
        assert FA.fekernel_name(O.kernel(name, "ref")) == name
    ref = lambda n: O.kernel(n, "ref")  # noqa: E731
    mesh = MESHES["tet4"]()
    mat = elastic_setup(mesh, seed=51)
    dm = FA.DeviceMesh(ctx, mesh)
    ig_lib = mat.create_integrator(dm)
    ig_ref = FA.IntegratorDomain(dm)
    for name, vals in (("density", mat.density), ("shear_modulus", mat.shear_modulus),
                       ("bulk_modulus", mat.bulk_modulus)):
        ig_ref.set_aux(name, FA.PER_CELL, vals[:, None])
    ig_ref.set_kernels_residual([FA.ResidualKernels("displacement", FA.LHS, None, ref(F1_ILE))])
    ig_ref.set_kernels_jacobian([FA.JacobianKernels("displacement", "displacement", FA.LHS, None, None, None,
                                                    ref(JF3_ILE))])
    u = dev(torch, np.random.default_rng(52).standard_normal(mesh.num_dof))
    outs = []
    for ig in (ig_lib, ig_ref):
        r, jv = torch.empty_like(u), torch.empty_like(u)
        ig.set_scatter(FA.SCATTER_DETERMINISTIC)
        ig.compute_lhs_residual(0.0, 0.0, u, r)
        ig.compute_lhs_jacobian_action(0.0, 0.0, 0.0, None, u, jv)
        outs.append((r, jv))
    ctx.synchronize()
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    # a fault with the reference's FaultCohesiveKin kernels
    fmesh, fault = fault_setup()
    fdm = FA.DeviceMesh(ctx, fmesh)
    if_lib = fault.create_integrator(fdm)
    if_ref = FA.IntegratorInterface(fdm)
    if_ref.set_aux("slip", FA.PER_FAULT_NODE, fault.slip)
    if_ref.set_constants(fault.constants)
    if_ref.set_kernels_residual([
        FA.InterfaceResidualKernels("displacement", FA.LHS, FA.FACE_NEGATIVE, ref("FaultCohesiveKin::f0u_neg"), None),
        FA.InterfaceResidualKernels("displacement", FA.LHS, FA.FACE_POSITIVE, ref("FaultCohesiveKin::f0u_pos"), None),
        FA.InterfaceResidualKernels("lagrange_multiplier_fault", FA.LHS, FA.FACE_FAULT,
                                    ref("FaultCohesiveKin::f0l_slip"), None)])
    fu = dev(torch, np.random.default_rng(53).standard_normal(fmesh.num_dof))
    fr = [torch.zeros_like(fu), torch.zeros_like(fu)]
    if_lib.compute_lhs_residual(0.0, 0.0, fu, fr[0])
    if_ref.compute_lhs_residual(0.0, 0.0, fu, fr[1])
    ctx.synchronize()
    assert torch.equal(fr[0], fr[1])
