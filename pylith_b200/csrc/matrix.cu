// Assembled Jacobian: 3x3-block CSR over the node graph (mesh nodes, then Lagrange nodes).
// Replaces the AIJ matrix PETSc fills with MatSetClosure inside DMPlexComputeJacobianByKey
// (IntegratorDomain.cc:489) and DMPlexComputeJacobianHybridByKey (IntegratorInterface.cc:714).
#include <algorithm>
#include <cstring>
#include <vector>

#include "domain_kernels.cuh"
#include "internal.hpp"
#include "launch.hpp"

using namespace plb;

namespace {

// y = A x for 3x3 blocks, one warp per block row.
__global__ void k_bsr_spmv(int64_t nrows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
    const int lane = threadIdx.x & 31;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < nrows;
         r += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        double a0 = 0.0, a1 = 0.0, a2 = 0.0;
        for (int k = rp[r] + lane; k < rp[r + 1]; k += 32) {
            const double* b = val + 9 * (int64_t)k;
            const int64_t c = ci[k];
            const double x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
            a0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
            a1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
            a2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_down_sync(0xffffffffu, a0, o);
            a1 += __shfl_down_sync(0xffffffffu, a1, o);
            a2 += __shfl_down_sync(0xffffffffu, a2, o);
        }
        if (lane == 0) {
            y[3 * r] = a0;
            y[3 * r + 1] = a1;
            y[3 * r + 2] = a2;
        }
    }
}

int find_block(const std::vector<int32_t>& rp, const std::vector<int32_t>& ci, int64_t r, int64_t c) {
    const int32_t* b = ci.data() + rp[r];
    const int32_t* e = ci.data() + rp[r + 1];
    const int32_t* it = std::lower_bound(b, e, (int32_t)c);
    return (it != e && *it == c) ? (int)(it - ci.data()) : -1;
}

}  // namespace

extern "C" {

int pl_matrix_create(pl_mesh m, pl_matrix* out) {
    if (!m || !out) return fail(PL_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    const int64_t nrows = m->nnodes + m->nlag;
    const int nen = m->nen;
    // pattern: pairs (row, col) as 64-bit keys
    std::vector<int64_t> keys;
    keys.reserve((size_t)m->ncells * nen * nen + (size_t)m->ncoh * 64 + nrows);
    for (int64_t r = 0; r < nrows; ++r) keys.push_back(r * nrows + r);
    for (int64_t c = 0; c < m->ncells; ++c) {
        const int32_t* cn = &m->h_cells[(size_t)c * nen];
        for (int a = 0; a < nen; ++a)
            for (int b = 0; b < nen; ++b) keys.push_back((int64_t)cn[a] * nrows + cn[b]);
    }
    for (int64_t c = 0; c < m->ncoh; ++c) {
        const int32_t* cc = &m->h_coh[(size_t)12 * c];
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const int64_t lb = m->nnodes + cc[8 + b], la = m->nnodes + cc[8 + a];
                keys.push_back((int64_t)cc[a] * nrows + lb);
                keys.push_back((int64_t)cc[4 + a] * nrows + lb);
                keys.push_back(la * nrows + cc[b]);
                keys.push_back(la * nrows + cc[4 + b]);
            }
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    if (keys.size() > (size_t)INT32_MAX) return fail(PL_ERR_UNSUPPORTED, "matrix too large for 32-bit block indices");
    std::vector<int32_t> rp(nrows + 1, 0), ci(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) {
        rp[keys[k] / nrows + 1]++;
        ci[k] = (int32_t)(keys[k] % nrows);
    }
    for (int64_t r = 0; r < nrows; ++r) rp[r + 1] += rp[r];
    std::vector<int32_t> cpos((size_t)m->ncells * nen * nen);
    for (int64_t c = 0; c < m->ncells; ++c) {
        const int32_t* cn = &m->h_cells[(size_t)c * nen];
        for (int a = 0; a < nen; ++a)
            for (int b = 0; b < nen; ++b)
                cpos[((size_t)c * nen + a) * nen + b] = find_block(rp, ci, cn[a], cn[b]);
    }
    std::vector<int32_t> hpos((size_t)m->ncoh * 64);
    for (int64_t c = 0; c < m->ncoh; ++c) {
        const int32_t* cc = &m->h_coh[(size_t)12 * c];
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) {
                const int64_t lb = m->nnodes + cc[8 + b], la = m->nnodes + cc[8 + a];
                hpos[(size_t)64 * c + (0 * 4 + a) * 4 + b] = find_block(rp, ci, cc[a], lb);
                hpos[(size_t)64 * c + (1 * 4 + a) * 4 + b] = find_block(rp, ci, cc[4 + a], lb);
                hpos[(size_t)64 * c + (2 * 4 + a) * 4 + b] = find_block(rp, ci, la, cc[b]);
                hpos[(size_t)64 * c + (3 * 4 + a) * 4 + b] = find_block(rp, ci, la, cc[4 + b]);
            }
    }
    for (int32_t v : cpos)
        if (v < 0) return fail(PL_ERR_INVALID_ARG, "internal: element block missing from the pattern");
    for (int32_t v : hpos)
        if (v < 0) return fail(PL_ERR_INVALID_ARG, "internal: cohesive block missing from the pattern");
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    pl_matrix A = new pl_matrix_s();
    A->mesh = m;
    mesh_retain(m);
    A->nrows = nrows;
    A->nnzb = (int64_t)ci.size();
    cudaStream_t s = m->ctx->stream;
    cudaError_t e = dev_alloc(&A->d_row_ptr, rp.size());
    if (e == cudaSuccess) e = dev_alloc(&A->d_col, ci.size());
    if (e == cudaSuccess) e = dev_alloc(&A->d_val, ci.size() * 9);
    if (e == cudaSuccess) e = dev_alloc(&A->d_cell_pos, cpos.size());
    if (e == cudaSuccess && !hpos.empty()) e = dev_alloc(&A->d_coh_pos, hpos.size());
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->d_row_ptr, rp.data(), rp.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->d_col, ci.data(), ci.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(A->d_cell_pos, cpos.data(), cpos.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && !hpos.empty())
        e = cudaMemcpyAsync(A->d_coh_pos, hpos.data(), hpos.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(A->d_val, 0, ci.size() * 9 * sizeof(double), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        pl_matrix_destroy(A);
        return cuda_fail(e, "pl_matrix_create");
    }
    *out = A;
    return PL_OK;
}

int pl_matrix_zero(pl_matrix A) {
    if (!A) return fail(PL_ERR_INVALID_ARG, "null matrix");
    PLB_CUDA(cudaSetDevice(A->mesh->ctx->device));
    PLB_CUDA(cudaMemsetAsync(A->d_val, 0, A->nnzb * 9 * sizeof(double), A->mesh->ctx->stream));
    return PL_OK;
}

int pl_compute_lhs_jacobian(pl_integrator ig, double t, double dt, double s_tshift, const double* u, pl_matrix A) {
    if (!ig || !A || A->mesh != ig->mesh) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    pl_mesh m = ig->mesh;
    cudaStream_t s = m->ctx->stream;
    PLB_CUDA(cudaSetDevice(m->ctx->device));
    if (ig->is_interface) {
        CohesiveParams p;
        std::memset(&p, 0, sizeof(p));
        p.coh = m->d_coh;
        p.ncoh = m->ncoh;
        p.coords = m->d_coords;
        p.lag_offset = 3 * m->nnodes;
        p.t = t;
        p.s_tshift = s_tshift;
        p.num_constants = (int)std::min<size_t>(ig->constants.size(), 8);
        for (int i = 0; i < p.num_constants; ++i) p.constants[i] = ig->constants[i];
        for (int f = 0; f < 3; ++f) p.kj[f] = ig->if_j[f];
        launch_cohesive_jacobian(p, A->d_coh_pos, A->d_val, s);
        PLB_CUDA(cudaGetLastError());
        return PL_OK;
    }
    if (ig->j3 == K_NONE) return fail(PL_ERR_NOT_READY, "no Jacobian kernels registered");
    DomainParams p;
    int rc = bind_domain_jacobian(ig, &p);
    if (rc) return rc;
    p.u = u;
    p.t = t;
    p.dt = dt;
    p.s_tshift = s_tshift;
    const int rheo = ig->j3 == K_ILE_JF3VU ? RHEO_ILE : RHEO_GENMAXWELL;
    launch_domain_jacobian(p, m->cell_type, rheo, A->d_cell_pos, A->d_val, s);
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_matrix_info(pl_matrix A, int64_t* nrows, int64_t* nnzb, const int32_t** rp, const int32_t** ci, double** val) {
    if (!A) return fail(PL_ERR_INVALID_ARG, "null matrix");
    if (nrows) *nrows = A->nrows;
    if (nnzb) *nnzb = A->nnzb;
    if (rp) *rp = A->d_row_ptr;
    if (ci) *ci = A->d_col;
    if (val) *val = A->d_val;
    return PL_OK;
}

int pl_matrix_copy_to_host(pl_matrix A, int32_t* rp, int32_t* ci, double* val) {
    if (!A || !rp || !ci || !val) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    cudaStream_t s = A->mesh->ctx->stream;
    PLB_CUDA(cudaSetDevice(A->mesh->ctx->device));
    PLB_CUDA(cudaMemcpyAsync(rp, A->d_row_ptr, (A->nrows + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaMemcpyAsync(ci, A->d_col, A->nnzb * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaMemcpyAsync(val, A->d_val, A->nnzb * 9 * sizeof(double), cudaMemcpyDeviceToHost, s));
    PLB_CUDA(cudaStreamSynchronize(s));
    return PL_OK;
}

int pl_matrix_spmv(pl_matrix A, const double* x, double* y) {
    if (!A || !x || !y) return fail(PL_ERR_INVALID_ARG, "bad arguments");
    PLB_CUDA(cudaSetDevice(A->mesh->ctx->device));
    const int64_t warps = A->nrows;
    int64_t blocks = (warps * 32 + 255) / 256;
    if (blocks > 148 * 32) blocks = 148 * 32;
    k_bsr_spmv<<<(int)std::max<int64_t>(blocks, 1), 256, 0, A->mesh->ctx->stream>>>(A->nrows, A->d_row_ptr, A->d_col, A->d_val, x, y);
    count_launch();
    PLB_CUDA(cudaGetLastError());
    return PL_OK;
}

int pl_matrix_destroy(pl_matrix A) {
    if (!A) return PL_OK;
    cudaSetDevice(A->mesh->ctx->device);
    cudaStreamSynchronize(A->mesh->ctx->stream);
    cudaStream_t s = A->mesh->ctx->stream;
    for (void* p : {(void*)A->d_row_ptr, (void*)A->d_col, (void*)A->d_val, (void*)A->d_cell_pos, (void*)A->d_coh_pos})
        dev_free(p, s);
    pl_mesh m = A->mesh;
    delete A;
    mesh_release(m);
    return PL_OK;
}

}  // extern "C"
