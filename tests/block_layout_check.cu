// Host check of the cell-block layout planner (plan_block in pylith_b200/csrc/blocked.cu), built
// by tests/test_block_layout.py: a Kuhn-split grid is cut into blocks of 256 cells, every block is
// planned, and the program prints one JSON line with the invariants (the local numbering is a
// permutation; every (cell, corner) appears once, under its node's new index) and the simulated
// shared-memory wavefronts of the corner gathers (FP64 node arrays: bank pair = local index mod 16)
// and of the per-node sums (bank pair = cell mod 16), with the nodes sorted by id and incidences in
// cell order, and with the planned layout. The pipelined kernel's incidence list must hold the same
// incidences per node, as staging offsets.
#include <cstdio>
#include <cstdlib>
#include <set>

#include "../pylith_b200/csrc/blocked.cu"

namespace plb {
void count_launch(int) {}
void ensure_kernel_smem(const void*, size_t) {}
int sm_count() { return 148; }
int cuda_fail(cudaError_t, const char*) { return PL_ERR_CUDA; }
int fail(int code, const std::string&) { return code; }
cudaError_t dev_alloc(void**, size_t) { return cudaErrorNotSupported; }
void dev_free(void*, cudaStream_t) {}
}  // namespace plb

using namespace plb;

static int wavefronts(const std::vector<int>& a) {
    std::set<int> u(a.begin(), a.end());
    int c[16] = {0}, m = 0;
    for (int x : u) m = std::max(m, ++c[x & 15]);
    return m;
}

int main(int argc, char** argv) {
    const int n = argc > 1 ? atoi(argv[1]) : 10;
    auto id = [&](int i, int j, int k) { return (i * (n + 1) + j) * (n + 1) + k; };
    const int perm[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    std::vector<int32_t> cells;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            for (int k = 0; k < n; ++k)
                for (const auto& p : perm) {
                    int x[3] = {i, j, k};
                    cells.push_back(id(x[0], x[1], x[2]));
                    for (int s = 0; s < 3; ++s) {
                        x[p[s]]++;
                        cells.push_back(id(x[0], x[1], x[2]));
                    }
                }
    const int64_t nc = (int64_t)cells.size() / 4, B = 256, nb = (nc + B - 1) / B;
    bool ok = true;
    long g0 = 0, g1 = 0, s0 = 0, s1 = 0, st0 = 0, st1 = 0;
    for (int64_t b = 0; b < nb; ++b) {
        const int ncell = (int)std::min<int64_t>(B, nc - b * B);
        const int32_t* bc = cells.data() + b * B * 4;
        BlockPlan P;
        plan_block(bc, ncell, (uint64_t)b, P);
        const int nloc = (int)P.loc.size();
        auto sorted_index = [&](int32_t node) {
            return (int)(std::lower_bound(P.loc.begin(), P.loc.end(), node) - P.loc.begin());
        };
        std::vector<int> seen(nloc, 0);
        for (int l = 0; l < nloc; ++l)
            ok = ok && P.newidx[l] >= 0 && P.newidx[l] < nloc && seen[P.newidx[l]]++ == 0;
        ok = ok && (int)P.off.size() == nloc + 1 && (int)P.inc.size() == 4 * ncell && P.off[nloc] == (uint32_t)(4 * ncell);
        if (!ok) break;
        std::vector<int> hit(4 * ncell, 0), hit_pipe(4 * ncell, 0);
        ok = ok && P.inc_pipe.size() == P.inc.size();
        for (int i = 0; ok && i < nloc; ++i)
            for (uint32_t j = P.off[i]; j < P.off[i + 1]; ++j) {
                const int e = P.inc[j];
                ok = ok && e < 4 * ncell && P.newidx[sorted_index(bc[e])] == i && hit[e]++ == 0;
                // the pipelined kernel's list: the same incidences of node i, as staging offsets
                // corner * 3 * 256 + cell
                const int q = P.inc_pipe[j], corner = q / (3 * 256), cell = q % (3 * 256);
                ok = ok && corner < 4 && cell < ncell && P.newidx[sorted_index(bc[4 * cell + corner])] == i &&
                     hit_pipe[4 * cell + corner]++ == 0;
            }
        for (int w = 0; w < ncell; w += 32)
            for (int k = 0; k < 4; ++k) {
                std::vector<int> a0, a1;
                for (int c = w; c < std::min(ncell, w + 32); ++c) {
                    const int l = sorted_index(bc[4 * c + k]);
                    a0.push_back(l);
                    a1.push_back(P.newidx[l]);
                }
                g0 += wavefronts(a0);
                g1 += wavefronts(a1);
            }
        std::vector<std::vector<int>> cell_order(nloc);
        for (int c = 0; c < ncell; ++c)
            for (int k = 0; k < 4; ++k) cell_order[sorted_index(bc[4 * c + k])].push_back(c);
        for (int w = 0; w < nloc; w += 32) {
            const int w1 = std::min(nloc, w + 32);
            size_t d0 = 0, d1 = 0;
            for (int i = w; i < w1; ++i) {
                d0 = std::max(d0, cell_order[i].size());
                d1 = std::max<size_t>(d1, P.off[i + 1] - P.off[i]);
            }
            st0 += (long)d0;
            st1 += (long)d1;
            for (size_t j = 0; j < d0; ++j) {
                std::vector<int> a;
                for (int i = w; i < w1; ++i)
                    if (j < cell_order[i].size()) a.push_back(cell_order[i][j]);
                s0 += wavefronts(a);
            }
            for (size_t j = 0; j < d1; ++j) {
                std::vector<int> a;
                for (int i = w; i < w1; ++i)
                    if (P.off[i] + j < P.off[i + 1]) a.push_back(P.inc[P.off[i] + j] >> 2);
                s1 += wavefronts(a);
            }
        }
    }
    printf("{\"ok\": %s, \"blocks\": %lld, \"gather\": [%ld, %ld], \"node_sums\": [%ld, %ld], \"steps\": [%ld, %ld]}\n",
           ok ? "true" : "false", (long long)nb, g0, g1, s0, s1, st0, st1);
    return ok ? 0 : 1;
}
