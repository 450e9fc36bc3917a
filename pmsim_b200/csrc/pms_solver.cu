// pms_solver.cu -- batched implicit Newton loop on the device: many independent problems held in
// one pms_elements handle (disjoint point/cell ranges), one element launch per Newton iteration for
// all of them, and each Newton system solved by a hand-written FP64 block-Jacobi PCG.
//
// Sequencing per problem follows SolverImplicit::iterate (reference src/fem/solver_implicit.rs:187-272)
// with the Lagrange-multiplier treatment of prescribed values (src/fem/bc_prescribed.rs:99-134):
// the augmented system [K A^T; A 0][mdu; mdl] = [F_int + A^T l; A u - c] is solved by elimination,
//   mdu_p = u_p - c,   K_ff mdu_f = R_f - K_fp mdu_p (PCG),   mdl = (R_p + l) - (K mdu)_p,
// which gives the same Newton iterates as the direct solve of the augmented system; the
// convergence tests (src/fem/convergence_control.rs:52-128) see the same quantities:
// max|R| over free rows, prescribed rows (R_p + l) and constraint rows (u_p - c), and
// rel(mdu) = max |mdu_i| / (1 + |mdu0_i|) over the DOFs and the multipliers.
//
// Determinism: every reduction is split into chunks that never straddle two problems; a chunk is
// reduced by a fixed tree and a problem sums its chunks in order, so a problem's results do not
// depend on which other problems share the batch (bit-identical alone and in the mix).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pms.h"
#include "pms_internal.h"

using namespace pms;

namespace {

constexpr int CHN = 128;  // nodes per reduction chunk (= threads per block of the node kernels)

struct SolverArgs {
    int nd;
    int64_t nnode, ndof;
    const int32_t* node_prob;    // problem of each node
    const int64_t* chunk_node0;  // first node of each chunk
    const int32_t* chunk_nnode;  // nodes in each chunk
    const int32_t* chunk_prob;   // problem of each chunk
    const int64_t* pchunk;       // chunks of problem p: [pchunk[p], pchunk[p+1])
    const int32_t* pres_idx;     // per DOF: index into the prescribed arrays, or -1
    const uint8_t* active;       // per problem: Newton iteration running
    uint8_t* pcg_active;         // per problem: PCG still iterating
};

__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = CHN / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] += sh[t + s];
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}
__device__ __forceinline__ double block_max(double v, double* sh) {
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int s = CHN / 2; s > 0; s >>= 1) {
        if (t < s) sh[t] = fmax(sh[t], sh[t + s]);
        __syncthreads();
    }
    const double r = sh[0];
    __syncthreads();
    return r;
}

// ---- Newton-level kernels ----------------------------------------------------------------

// Residual rows (R = F_int - F_ext, R_p + l, u_p - c) and their per-chunk max-abs.
__global__ void residual_kernel(SolverArgs S, const double* ff, const double* fext, const double* u,
                                const double* lam, const double* c, double* rr, double* part_max) {
    __shared__ double sh[CHN];
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    double m = 0.0;
    if (S.active[pr] && threadIdx.x < S.chunk_nnode[ch]) {
        const int64_t node = S.chunk_node0[ch] + threadIdx.x;
        for (int d = 0; d < S.nd; d++) {
            const int64_t i = node * S.nd + d;
            double v = ff[i] - (fext ? fext[i] : 0.0);
            const int k = S.pres_idx[i];
            if (k >= 0) {
                v += lam[k];
                const double g = u[i] - c[k];
                m = fmax(m, isfinite(g) ? fabs(g) : INFINITY);
            }
            rr[i] = v;
            m = fmax(m, isfinite(v) ? fabs(v) : INFINITY);
        }
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) part_max[ch] = m;
}

// per problem: max over its chunks (op 0), sum (op 1)
__global__ void finalize_kernel(int np, const int64_t* pchunk, const double* part, double* out, int op) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    double v = 0.0;
    for (int64_t c = pchunk[p]; c < pchunk[p + 1]; c++) v = (op == 0) ? fmax(v, part[c]) : v + part[c];
    out[p] = v;
}

// Inverse of the free part of each node's diagonal block (block-Jacobi preconditioner).
__global__ void block_jacobi_kernel(SolverArgs S, const int64_t* bptr, const int32_t* kdiag, const double* csr,
                                    double* binv) {
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= S.nnode) return;
    if (!S.active[S.node_prob[node]]) return;
    const int nd = S.nd;
    const int64_t b0 = bptr[node], nb = bptr[node + 1] - b0;
    const int64_t base = (int64_t)nd * nd * b0 + (int64_t)kdiag[node] * nd;
    double a[3][6];
    int fr[3], nf = 0;
    for (int i = 0; i < nd; i++)
        if (S.pres_idx[node * nd + i] < 0) fr[nf++] = i;
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) {
            a[i][j] = csr[base + (int64_t)fr[i] * nd * nb + fr[j]];
            a[i][nf + j] = (i == j) ? 1.0 : 0.0;
        }
    // Gauss-Jordan without pivoting: the diagonal block of an SPD matrix is SPD
    bool ok = true;
    for (int k = 0; k < nf; k++) {
        const double piv = a[k][k];
        if (!(piv > 0.0)) { ok = false; break; }
        const double ip = 1.0 / piv;
        for (int j = 0; j < 2 * nf; j++) a[k][j] *= ip;
        for (int i = 0; i < nf; i++)
            if (i != k) {
                const double f = a[i][k];
                for (int j = 0; j < 2 * nf; j++) a[i][j] -= f * a[k][j];
            }
    }
    double* out = binv + node * nd * nd;
    for (int i = 0; i < nd * nd; i++) out[i] = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) out[fr[i] * nd + fr[j]] = ok ? a[i][nf + j] : (i == j ? 1.0 / fmax(fabs(a[i][i]), 1e-300) : 0.0);
}

// y = K x on the rows of active problems (tpr threads per row); masked: y_p = 0 on prescribed rows
// when mask_pres, and only problems with flag[p] set take part.
template <int TPR>
__global__ void spmv_kernel(SolverArgs S, const int64_t* indptr, const int32_t* indices, const double* val,
                            const double* x, double* y, const uint8_t* flag, bool mask_pres) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t row = gid / TPR;
    const int sub = (int)(gid % TPR);
    // no early exit: every lane of the warp takes part in the shuffles below
    const bool on = row < S.ndof && flag[S.node_prob[row < S.ndof ? row / S.nd : 0]];
    double s = 0.0;
    if (on)
        for (int64_t k = indptr[row] + sub; k < indptr[row + 1]; k += TPR) s = fma(val[k], x[indices[k]], s);
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, TPR);
    if (on && sub == 0) y[row] = (mask_pres && S.pres_idx[row] >= 0) ? 0.0 : s;
}

// mdu_p = u_p - c on prescribed rows (0 elsewhere), for active problems
__global__ void pres_increment_kernel(SolverArgs S, const double* u, const double* c, double* mdu) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ndof) return;
    if (!S.active[S.node_prob[i / S.nd]]) return;
    const int k = S.pres_idx[i];
    mdu[i] = (k >= 0) ? u[i] - c[k] : 0.0;
}

// PCG start: r = R_f - (K mdu_p)_f, x = 0, z = M r, p = z; partials of r.z and r.r
__global__ void pcg_start_kernel(SolverArgs S, const double* rr, const double* kt, const double* binv, double* r,
                                 double* x, double* z, double* p, double* part_rz, double* part_rr) {
    __shared__ double sh[CHN];
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    double rz = 0.0, r2 = 0.0;
    const bool on = S.active[pr] && threadIdx.x < S.chunk_nnode[ch];
    if (on) {
        const int64_t node = S.chunk_node0[ch] + threadIdx.x;
        const int nd = S.nd;
        double rv[3];
        for (int d = 0; d < nd; d++) {
            const int64_t i = node * nd + d;
            rv[d] = (S.pres_idx[i] >= 0) ? 0.0 : rr[i] - kt[i];
            r[i] = rv[d];
            x[i] = 0.0;
        }
        const double* B = binv + node * nd * nd;
        for (int d = 0; d < nd; d++) {
            double zv = 0.0;
            for (int e = 0; e < nd; e++) zv += B[d * nd + e] * rv[e];
            z[node * nd + d] = zv;
            p[node * nd + d] = zv;
            rz += rv[d] * zv;
            r2 += rv[d] * rv[d];
        }
    }
    rz = block_sum(rz, sh);
    r2 = block_sum(r2, sh);
    if (threadIdx.x == 0) {
        part_rz[ch] = rz;
        part_rr[ch] = r2;
    }
}

__global__ void pcg_init_scalars_kernel(int np, const uint8_t* active, const int64_t* pchunk, const double* part_rz,
                                        const double* part_rr, double* rho, double* r0, uint8_t* pcg_active,
                                        int32_t* pcg_iters) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    double a = 0.0, b = 0.0;
    for (int64_t c = pchunk[p]; c < pchunk[p + 1]; c++) {
        a += part_rz[c];
        b += part_rr[c];
    }
    rho[p] = a;
    r0[p] = sqrt(b);
    pcg_active[p] = (active[p] && b > 0.0) ? 1 : 0;
    pcg_iters[p] = 0;
}

// partials of p.q
__global__ void pcg_dot_kernel(SolverArgs S, const double* a, const double* b, double* part) {
    __shared__ double sh[CHN];
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    double s = 0.0;
    if (S.pcg_active[pr] && threadIdx.x < S.chunk_nnode[ch]) {
        const int64_t node = S.chunk_node0[ch] + threadIdx.x;
        for (int d = 0; d < S.nd; d++) {
            const int64_t i = node * S.nd + d;
            if (S.pres_idx[i] < 0) s += a[i] * b[i];
        }
    }
    s = block_sum(s, sh);
    if (threadIdx.x == 0) part[ch] = s;
}

__global__ void pcg_alpha_kernel(int np, const uint8_t* pcg_active, const int64_t* pchunk, const double* part,
                                 const double* rho, double* alpha) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    double pq = 0.0;
    for (int64_t c = pchunk[p]; c < pchunk[p + 1]; c++) pq += part[c];
    alpha[p] = (pcg_active[p] && pq != 0.0) ? rho[p] / pq : 0.0;
}

// x += a p, r -= a q, z = M r; partials of r.z and r.r
__global__ void pcg_update_kernel(SolverArgs S, const double* alpha, const double* p, const double* q,
                                  const double* binv, double* x, double* r, double* z, double* part_rz,
                                  double* part_rr) {
    __shared__ double sh[CHN];
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    double rz = 0.0, r2 = 0.0;
    if (S.pcg_active[pr] && threadIdx.x < S.chunk_nnode[ch]) {
        const int64_t node = S.chunk_node0[ch] + threadIdx.x;
        const int nd = S.nd;
        const double a = alpha[pr];
        double rv[3];
        for (int d = 0; d < nd; d++) {
            const int64_t i = node * nd + d;
            if (S.pres_idx[i] < 0) {
                x[i] += a * p[i];
                rv[d] = r[i] - a * q[i];
                r[i] = rv[d];
            } else {
                rv[d] = 0.0;
            }
        }
        const double* B = binv + node * nd * nd;
        for (int d = 0; d < nd; d++) {
            double zv = 0.0;
            for (int e = 0; e < nd; e++) zv += B[d * nd + e] * rv[e];
            z[node * nd + d] = zv;
            rz += rv[d] * zv;
            r2 += rv[d] * rv[d];
        }
    }
    rz = block_sum(rz, sh);
    r2 = block_sum(r2, sh);
    if (threadIdx.x == 0) {
        part_rz[ch] = rz;
        part_rr[ch] = r2;
    }
}

__global__ void pcg_beta_kernel(int np, uint8_t* pcg_active, const int64_t* pchunk, const double* part_rz,
                                const double* part_rr, double* rho, double* beta, const double* r0, double rtol,
                                int32_t max_iter, int32_t* iters, int32_t* nactive) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    if (!pcg_active[p]) {
        beta[p] = 0.0;
        return;
    }
    double a = 0.0, b = 0.0;
    for (int64_t c = pchunk[p]; c < pchunk[p + 1]; c++) {
        a += part_rz[c];
        b += part_rr[c];
    }
    beta[p] = (rho[p] != 0.0) ? a / rho[p] : 0.0;
    rho[p] = a;
    iters[p] += 1;
    const bool done = !(sqrt(b) > rtol * r0[p]) || iters[p] >= max_iter;
    if (done) {
        pcg_active[p] = 0;
    } else {
        atomicAdd(nactive, 1);
    }
}

__global__ void pcg_p_kernel(SolverArgs S, const uint8_t* was_active, const double* beta, const double* z,
                             double* p) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ndof) return;
    const int pr = S.node_prob[i / S.nd];
    if (!was_active[pr]) return;
    p[i] = (S.pres_idx[i] >= 0) ? 0.0 : z[i] + beta[pr] * p[i];
}

// mdu = x on free rows (mdu already holds u_p - c on prescribed rows); mdl = (R_p + l) - (K mdu)_p
__global__ void assemble_mdu_kernel(SolverArgs S, const double* x, double* mdu) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ndof) return;
    if (!S.active[S.node_prob[i / S.nd]]) return;
    if (S.pres_idx[i] < 0) mdu[i] = x[i];
}

__global__ void multiplier_kernel(int64_t npres, const int64_t* pres_eq, const int32_t* pres_prob,
                                  const uint8_t* active, const int64_t* indptr, const int32_t* indices,
                                  const double* val, const double* mdu, const double* rr, double* mdl) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npres) return;
    if (!active[pres_prob[k]]) return;
    const int64_t row = pres_eq[k];
    double s = 0.0;
    for (int64_t j = indptr[row]; j < indptr[row + 1]; j++) s = fma(val[j], mdu[indices[j]], s);
    mdl[k] = rr[row] - s;  // rr[row] already holds R_p + l
}

// rel(mdu) partials: max |mdu_i| / (1 + |mdu0_i|) over DOFs (it > 0), or save mdu0 (it == 0)
__global__ void rel_mdu_kernel(SolverArgs S, const uint8_t* first, const double* mdu, double* mdu0,
                               double* part_max) {
    __shared__ double sh[CHN];
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    double m = 0.0;
    if (S.active[pr] && threadIdx.x < S.chunk_nnode[ch]) {
        const int64_t node = S.chunk_node0[ch] + threadIdx.x;
        for (int d = 0; d < S.nd; d++) {
            const int64_t i = node * S.nd + d;
            const double v = mdu[i];
            if (first[pr]) {
                mdu0[i] = v;
                m = fmax(m, isfinite(v) ? 0.0 : INFINITY);
            } else {
                const double r = fabs(v) / (1.0 + fabs(mdu0[i]));
                m = fmax(m, isfinite(r) ? r : INFINITY);
            }
        }
    }
    m = block_max(m, sh);
    if (threadIdx.x == 0) part_max[ch] = m;
}

// per problem: fold the multiplier entries into rel(mdu); save mdl0 at the first iteration
__global__ void rel_multipliers_kernel(int np, const uint8_t* active, const uint8_t* first, const int64_t* ppres,
                                       const double* mdl, double* mdl0, double* rel) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np || !active[p]) return;
    double m = rel[p];
    for (int64_t k = ppres[p]; k < ppres[p + 1]; k++) {
        if (first[p]) {
            mdl0[k] = mdl[k];
            if (!isfinite(mdl[k])) m = INFINITY;
        } else {
            const double r = fabs(mdl[k]) / (1.0 + fabs(mdl0[k]));
            m = fmax(m, isfinite(r) ? r : INFINITY);
        }
    }
    rel[p] = first[p] ? (isfinite(m) ? 1.0 : INFINITY) : m;
}

// U -= mdu, dU -= mdu on every unknown (LMM: all equations), l -= mdl
__global__ void update_kernel(SolverArgs S, const uint8_t* upd, const double* mdu, double* u, double* ddu) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ndof) return;
    if (!upd[S.node_prob[i / S.nd]]) return;
    u[i] -= mdu[i];
    ddu[i] -= mdu[i];
}

__global__ void update_multipliers_kernel(int64_t npres, const int32_t* pres_prob, const uint8_t* upd,
                                          const double* mdl, double* lam) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= npres) return;
    if (upd[pres_prob[k]]) lam[k] -= mdl[k];
}

__global__ void zero_masked_kernel(SolverArgs S, const uint8_t* flag, double* v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ndof) return;
    if (flag[S.node_prob[i / S.nd]]) v[i] = 0.0;
}

}  // namespace

// ------------------------------------------------------------------------------------ handle
struct pms_batch {
    pms_elements* el = nullptr;
    ElementsView v{};
    int np = 0;
    int64_t nnode = 0, ndof = 0, npres = 0, nchunk = 0;
    pms_batch_config cfg{};
    std::vector<int64_t> point_ptr, cell_ptr, pres_ptr;
    std::vector<void*> allocs;
    // device
    int32_t *d_node_prob = nullptr, *d_cell_prob = nullptr, *d_chunk_nnode = nullptr, *d_chunk_prob = nullptr;
    int64_t *d_chunk_node0 = nullptr, *d_pchunk = nullptr, *d_ppres = nullptr, *d_pres_eq = nullptr;
    int32_t *d_pres_idx = nullptr, *d_pres_prob = nullptr;
    uint8_t *d_active = nullptr, *d_pcg_active = nullptr, *d_pcg_was = nullptr, *d_pmode = nullptr,
            *d_first = nullptr, *d_upd = nullptr;
    double *d_u = nullptr, *d_ddu = nullptr, *d_ff = nullptr, *d_fext = nullptr, *d_csr = nullptr, *d_rr = nullptr;
    double *d_mdu = nullptr, *d_mdu0 = nullptr, *d_kt = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr,
           *d_q = nullptr, *d_x = nullptr, *d_binv = nullptr;
    double *d_lam = nullptr, *d_c = nullptr, *d_mdl = nullptr, *d_mdl0 = nullptr;
    double *d_part_a = nullptr, *d_part_b = nullptr;
    double *d_rho = nullptr, *d_r0 = nullptr, *d_alpha = nullptr, *d_beta = nullptr, *d_norm = nullptr,
           *d_rel = nullptr;
    int32_t *d_iters = nullptr, *d_nactive = nullptr;
    const int64_t* d_indptr = nullptr;
    const int32_t* d_indices = nullptr;
    SolverArgs S{};
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    std::string last_error;
    int64_t launches = 0;
    int64_t pcg_total = 0;
    std::vector<int32_t> it;  // Newton iteration of each problem within its current load step

    template <typename T>
    bool alloc(T** p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        std::lock_guard<std::mutex> lock(device_mutex());
        if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) return false;
        allocs.push_back((void*)*p);
        return true;
    }
    template <typename T>
    bool upload(T** p, const T* src, size_t count) {
        if (!alloc(p, count)) return false;
        return count == 0 || cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
    }
    ~pms_batch() {
        cudaStreamSynchronize(v.stream);
        std::lock_guard<std::mutex> lock(device_mutex());
        if (graph) cudaGraphExecDestroy(graph);
        for (void* p : allocs) cudaFree(p);
    }
};

namespace {

int bfail(pms_batch* b, int code, const char* msg) {
    if (b) b->last_error = msg;
    return code;
}

inline unsigned grid_of(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>((n + t - 1) / t, 1); }

void launch_spmv(pms_batch* b, const double* x, double* y, const uint8_t* flag, bool mask) {
    const int tpr = b->v.nd == 2 ? 8 : 16;
    const int64_t threads = b->ndof * tpr;
    if (tpr == 8)
        spmv_kernel<8><<<grid_of(threads), 256, 0, b->v.stream>>>(b->S, b->d_indptr, b->d_indices, b->d_csr, x, y,
                                                                   flag, mask);
    else
        spmv_kernel<16><<<grid_of(threads), 256, 0, b->v.stream>>>(b->S, b->d_indptr, b->d_indices, b->d_csr, x, y,
                                                                    flag, mask);
    b->launches++;
}

// one PCG iteration for every problem with pcg_active set
void pcg_iteration(pms_batch* b) {
    cudaStream_t st = b->v.stream;
    const int np = b->np;
    const unsigned gp = grid_of(np, 128);
    cudaMemsetAsync(b->d_nactive, 0, sizeof(int32_t), st);  // counts the problems still active after this iteration
    cudaMemcpyAsync(b->d_pcg_was, b->d_pcg_active, np, cudaMemcpyDeviceToDevice, st);
    launch_spmv(b, b->d_p, b->d_q, b->d_pcg_active, true);
    pcg_dot_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_p, b->d_q, b->d_part_a);
    pcg_alpha_kernel<<<gp, 128, 0, st>>>(np, b->d_pcg_active, b->d_pchunk, b->d_part_a, b->d_rho, b->d_alpha);
    pcg_update_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_alpha, b->d_p, b->d_q, b->d_binv, b->d_x,
                                                           b->d_r, b->d_z, b->d_part_a, b->d_part_b);
    pcg_beta_kernel<<<gp, 128, 0, st>>>(np, b->d_pcg_active, b->d_pchunk, b->d_part_a, b->d_part_b, b->d_rho,
                                        b->d_beta, b->d_r0, b->cfg.pcg_rtol, b->cfg.pcg_max_iterations, b->d_iters,
                                        b->d_nactive);
    pcg_p_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_pcg_was, b->d_beta, b->d_z, b->d_p);
    b->launches += 5;
}

// PCG until every problem has converged (or reached the iteration cap); iterations run in CUDA
// graphs of graph_iters iterations between host checks of the number of active problems.
int run_pcg(pms_batch* b) {
    cudaStream_t st = b->v.stream;
    if (!b->graph) {
        std::lock_guard<std::mutex> lock(device_mutex());
        cudaGraph_t g;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return bfail(b, PMS_ERR_CUDA, "stream capture failed");
        for (int i = 0; i < b->graph_iters; i++) pcg_iteration(b);
        if (cudaStreamEndCapture(st, &g) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "stream capture failed");
        if (cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) {
            cudaGraphDestroy(g);
            return bfail(b, PMS_ERR_CUDA, "graph instantiation failed");
        }
        cudaGraphDestroy(g);
    }
    int32_t nact = 1;
    for (int64_t it = 0; it < b->cfg.pcg_max_iterations && nact > 0; it += b->graph_iters) {
        if (cudaGraphLaunch(b->graph, st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "graph launch failed");
        cudaMemcpyAsync(&nact, b->d_nactive, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    }
    return PMS_OK;
}

}  // namespace

extern "C" {

int pms_batch_create(pms_elements* el, int32_t nproblem, const int64_t* point_ptr, const int64_t* cell_ptr,
                     int64_t npres, const int64_t* pres_eq, const double* ff_ext, const pms_batch_config* cfg,
                     pms_batch** out) {
    if (!out) return PMS_ERR_INVALID;
    *out = nullptr;
    if (!el || nproblem < 1 || !point_ptr || !cell_ptr || npres < 0 || (npres > 0 && !pres_eq) || !cfg)
        return PMS_ERR_INVALID;
    auto* b = new pms_batch();
    b->el = el;
    b->v = elements_view(el);
    b->np = nproblem;
    b->nnode = b->v.npoint;
    b->ndof = b->v.ndof;
    b->npres = npres;
    b->cfg = *cfg;
    if (b->cfg.pcg_max_iterations <= 0) b->cfg.pcg_max_iterations = 20000;
    if (!(b->cfg.pcg_rtol > 0)) b->cfg.pcg_rtol = 1e-12;
    if (b->cfg.n_max_iterations <= 0) b->cfg.n_max_iterations = 10;
    b->graph_iters = 8;
    const int nd = b->v.nd;
    b->point_ptr.assign(point_ptr, point_ptr + nproblem + 1);
    b->cell_ptr.assign(cell_ptr, cell_ptr + nproblem + 1);
    if (point_ptr[0] != 0 || point_ptr[nproblem] != b->nnode || cell_ptr[0] != 0 || cell_ptr[nproblem] != b->v.ncell) {
        delete b;
        return PMS_ERR_INVALID;
    }
    for (int p = 0; p < nproblem; p++)
        if (point_ptr[p + 1] < point_ptr[p] || cell_ptr[p + 1] < cell_ptr[p]) {
            delete b;
            return PMS_ERR_INVALID;
        }
    // per node / per cell problem ids, reduction chunks
    std::vector<int32_t> node_prob(b->nnode), cell_prob(b->v.ncell);
    std::vector<int64_t> chunk_node0, pchunk(nproblem + 1, 0);
    std::vector<int32_t> chunk_nnode, chunk_prob;
    for (int p = 0; p < nproblem; p++) {
        for (int64_t i = point_ptr[p]; i < point_ptr[p + 1]; i++) node_prob[i] = p;
        for (int64_t c = cell_ptr[p]; c < cell_ptr[p + 1]; c++) cell_prob[c] = p;
        pchunk[p] = (int64_t)chunk_node0.size();
        for (int64_t i = point_ptr[p]; i < point_ptr[p + 1]; i += CHN) {
            chunk_node0.push_back(i);
            chunk_nnode.push_back((int32_t)std::min<int64_t>(CHN, point_ptr[p + 1] - i));
            chunk_prob.push_back(p);
        }
    }
    pchunk[nproblem] = (int64_t)chunk_node0.size();
    b->nchunk = (int64_t)chunk_node0.size();
    // prescribed equations (sorted, unique), their problems and per-problem ranges
    std::vector<int64_t> peq(pres_eq, pres_eq + npres);
    for (int64_t k = 1; k < npres; k++)
        if (peq[k] <= peq[k - 1]) {
            delete b;
            return PMS_ERR_INVALID;  // must be sorted and unique
        }
    std::vector<int32_t> pres_idx(b->ndof, -1), pres_prob(npres);
    b->pres_ptr.assign(nproblem + 1, 0);
    for (int64_t k = 0; k < npres; k++) {
        if (peq[k] < 0 || peq[k] >= b->ndof) {
            delete b;
            return PMS_ERR_INVALID;
        }
        pres_idx[peq[k]] = (int32_t)k;
        pres_prob[k] = node_prob[peq[k] / nd];
        b->pres_ptr[pres_prob[k] + 1]++;
    }
    for (int p = 0; p < nproblem; p++) b->pres_ptr[p + 1] += b->pres_ptr[p];
    const size_t n = (size_t)b->ndof;
    bool ok = b->upload(&b->d_node_prob, node_prob.data(), node_prob.size()) &&
              b->upload(&b->d_cell_prob, cell_prob.data(), cell_prob.size()) &&
              b->upload(&b->d_chunk_node0, chunk_node0.data(), chunk_node0.size()) &&
              b->upload(&b->d_chunk_nnode, chunk_nnode.data(), chunk_nnode.size()) &&
              b->upload(&b->d_chunk_prob, chunk_prob.data(), chunk_prob.size()) &&
              b->upload(&b->d_pchunk, pchunk.data(), pchunk.size()) &&
              b->upload(&b->d_ppres, b->pres_ptr.data(), b->pres_ptr.size()) &&
              b->upload(&b->d_pres_eq, peq.data(), peq.size()) &&
              b->upload(&b->d_pres_idx, pres_idx.data(), pres_idx.size()) &&
              b->upload(&b->d_pres_prob, pres_prob.data(), pres_prob.size()) &&
              b->alloc(&b->d_active, nproblem) && b->alloc(&b->d_pcg_active, nproblem) &&
              b->alloc(&b->d_pcg_was, nproblem) && b->alloc(&b->d_pmode, nproblem) &&
              b->alloc(&b->d_first, nproblem) && b->alloc(&b->d_upd, nproblem) && b->alloc(&b->d_u, n) &&
              b->alloc(&b->d_ddu, n) && b->alloc(&b->d_ff, n) && b->alloc(&b->d_csr, (size_t)b->v.nnz) &&
              b->alloc(&b->d_rr, n) && b->alloc(&b->d_mdu, n) && b->alloc(&b->d_mdu0, n) &&
              b->alloc(&b->d_kt, n) && b->alloc(&b->d_r, n) && b->alloc(&b->d_z, n) && b->alloc(&b->d_p, n) &&
              b->alloc(&b->d_q, n) && b->alloc(&b->d_x, n) && b->alloc(&b->d_binv, (size_t)b->nnode * nd * nd) &&
              b->alloc(&b->d_lam, npres) && b->alloc(&b->d_c, npres) && b->alloc(&b->d_mdl, npres) &&
              b->alloc(&b->d_mdl0, npres) && b->alloc(&b->d_part_a, b->nchunk) && b->alloc(&b->d_part_b, b->nchunk) &&
              b->alloc(&b->d_rho, nproblem) && b->alloc(&b->d_r0, nproblem) && b->alloc(&b->d_alpha, nproblem) &&
              b->alloc(&b->d_beta, nproblem) && b->alloc(&b->d_norm, nproblem) && b->alloc(&b->d_rel, nproblem) &&
              b->alloc(&b->d_iters, nproblem) && b->alloc(&b->d_nactive, 1);
    if (ok && ff_ext) ok = b->upload(&b->d_fext, ff_ext, n);
    if (!ok) {
        delete b;
        return PMS_ERR_NOMEM;
    }
    int rc = elements_device_pattern(el, &b->d_indptr, &b->d_indices);
    if (rc) {
        delete b;
        return rc;
    }
    cudaMemset(b->d_u, 0, n * 8);
    cudaMemset(b->d_ddu, 0, n * 8);
    cudaMemset(b->d_lam, 0, std::max<int64_t>(npres, 1) * 8);
    cudaMemset(b->d_p, 0, n * 8);
    b->S.nd = nd;
    b->S.nnode = b->nnode;
    b->S.ndof = b->ndof;
    b->S.node_prob = b->d_node_prob;
    b->S.chunk_node0 = b->d_chunk_node0;
    b->S.chunk_nnode = b->d_chunk_nnode;
    b->S.chunk_prob = b->d_chunk_prob;
    b->S.pchunk = b->d_pchunk;
    b->S.pres_idx = b->d_pres_idx;
    b->S.active = b->d_active;
    b->S.pcg_active = b->d_pcg_active;
    if (cudaDeviceSynchronize() != cudaSuccess) {
        delete b;
        return PMS_ERR_CUDA;
    }
    *out = b;
    return PMS_OK;
}

void pms_batch_destroy(pms_batch* b) { delete b; }

int pms_batch_reset(pms_batch* b) {
    if (!b) return PMS_ERR_INVALID;
    cudaStream_t st = b->v.stream;
    cudaMemsetAsync(b->d_u, 0, b->ndof * 8, st);
    cudaMemsetAsync(b->d_ddu, 0, b->ndof * 8, st);
    cudaMemsetAsync(b->d_lam, 0, std::max<int64_t>(b->npres, 1) * 8, st);
    int rc = pms_elements_initialize(b->el);
    if (rc) return rc;
    return cudaStreamSynchronize(st) == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}

int pms_batch_tick(pms_batch* b, const uint8_t* cmd, const double* c_values, int32_t* result, int32_t* iteration,
                   double* norm_rr, int32_t* pcg_iterations) {
    if (!b || !cmd || !result) return PMS_ERR_INVALID;
    if (b->npres > 0 && !c_values) return PMS_ERR_INVALID;
    cudaStream_t st = b->v.stream;
    const int np = b->np;
    std::vector<uint8_t> running(np, 0), mode(np, 0), first(np, 0), upd(np, 0), start(np, 0);
    std::vector<int32_t> pcg_step(np, 0);
    std::vector<double> hnorm(np, 0.0), hrel(np, 0.0);
    if ((int)b->it.size() != np) b->it.assign(np, 0);
    for (int p = 0; p < np; p++) {
        result[p] = -1;
        if (cmd[p] == 1) {
            b->it[p] = 0;
            start[p] = 1;
        }
        running[p] = cmd[p] != 0;
        mode[p] = cmd[p] == 1 ? 1 : (cmd[p] == 2 ? 2 : 0);
    }
    if (b->npres > 0) cudaMemcpyAsync(b->d_c, c_values, b->npres * 8, cudaMemcpyHostToDevice, st);
    // a new load step: dU = 0 (the loading time t += dt is in c_values)
    cudaMemcpyAsync(b->d_upd, start.data(), np, cudaMemcpyHostToDevice, st);
    zero_masked_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_upd, b->d_ddu);
    // element pass: step start (assemble with lambda = 0, backup) or stress update + assemble
    cudaMemcpyAsync(b->d_pmode, mode.data(), np, cudaMemcpyHostToDevice, st);
    int rc = elements_run_modes(b->el, b->d_cell_prob, b->d_node_prob, b->d_pmode, b->d_ddu, b->d_ff, b->d_csr);
    if (rc) return rc;
    // residual and its max norm per problem
    cudaMemcpyAsync(b->d_active, running.data(), np, cudaMemcpyHostToDevice, st);
    residual_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_ff, b->d_fext, b->d_u, b->d_lam, b->d_c, b->d_rr,
                                                         b->d_part_a);
    finalize_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_pchunk, b->d_part_a, b->d_norm, 0);
    cudaMemcpyAsync(hnorm.data(), b->d_norm, np * 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "residual failed");
    // a material or geometry error in one problem stops that problem only
    rc = elements_status(b->el);
    if (rc == PMS_ERR_ZERO_SIGMA_D || rc == PMS_ERR_ZERO_NORM_S || rc == PMS_ERR_JACOBIAN) {
        int64_t cell = -1;
        int32_t ip = -1;
        pms_elements_error_location(b->el, &cell, &ip);
        const int p = (int)(std::upper_bound(b->cell_ptr.begin(), b->cell_ptr.end(), cell) - b->cell_ptr.begin()) - 1;
        if (p >= 0 && p < np && running[p]) {
            result[p] = 100 + 1 + rc;  // 104: zero sigma_d, 105: zero norm_s, 106: Jacobian
            running[p] = 0;
        }
    } else if (rc) {
        return rc;
    }
    bool any = false;
    for (int p = 0; p < np; p++) {
        if (!running[p]) continue;
        if (iteration) iteration[p] = b->it[p];
        if (norm_rr) norm_rr[p] = hnorm[p];
        if (!std::isfinite(hnorm[p])) {
            result[p] = 101;  // "Found NaN or Inf"
            running[p] = 0;
        } else if (hnorm[p] < b->cfg.tol_rr_abs) {
            result[p] = 1;
            running[p] = 0;
        }
        any = any || running[p];
    }
    if (any) {
        // linear solve (mdu, mdl) for the problems still iterating
        cudaMemcpyAsync(b->d_active, running.data(), np, cudaMemcpyHostToDevice, st);
        block_jacobi_kernel<<<grid_of(b->nnode), 256, 0, st>>>(b->S, b->v.d_bptr, b->v.d_kdiag, b->d_csr, b->d_binv);
        pres_increment_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_u, b->d_c, b->d_mdu);
        launch_spmv(b, b->d_mdu, b->d_kt, b->d_active, false);
        pcg_start_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_rr, b->d_kt, b->d_binv, b->d_r, b->d_x,
                                                               b->d_z, b->d_p, b->d_part_a, b->d_part_b);
        pcg_init_scalars_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_active, b->d_pchunk, b->d_part_a,
                                                                   b->d_part_b, b->d_rho, b->d_r0, b->d_pcg_active,
                                                                   b->d_iters);
        rc = run_pcg(b);
        if (rc) return rc;
        cudaMemcpyAsync(pcg_step.data(), b->d_iters, np * 4, cudaMemcpyDeviceToHost, st);
        assemble_mdu_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_x, b->d_mdu);
        if (b->npres > 0)
            multiplier_kernel<<<grid_of(b->npres), 256, 0, st>>>(b->npres, b->d_pres_eq, b->d_pres_prob, b->d_active,
                                                                  b->d_indptr, b->d_indices, b->d_csr, b->d_mdu,
                                                                  b->d_rr, b->d_mdl);
        for (int p = 0; p < np; p++) first[p] = (b->it[p] == 0);
        cudaMemcpyAsync(b->d_first, first.data(), np, cudaMemcpyHostToDevice, st);
        rel_mdu_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_first, b->d_mdu, b->d_mdu0, b->d_part_a);
        finalize_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_pchunk, b->d_part_a, b->d_rel, 0);
        rel_multipliers_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_active, b->d_first, b->d_ppres, b->d_mdl,
                                                                  b->d_mdl0, b->d_rel);
        cudaMemcpyAsync(hrel.data(), b->d_rel, np * 8, cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "solve failed");
        for (int p = 0; p < np; p++) {
            upd[p] = 0;
            if (!running[p]) continue;
            if (pcg_iterations) pcg_iterations[p] = pcg_step[p];
            b->pcg_total += pcg_step[p];
            if (!std::isfinite(hrel[p])) {
                result[p] = 102;  // "Found NaN or Inf in mdu"
            } else if (b->it[p] > 0 && hrel[p] < b->cfg.tol_mdu_rel) {
                result[p] = 1;  // converged without applying this correction
            } else {
                upd[p] = 1;
                b->it[p] += 1;
                result[p] = (b->it[p] >= b->cfg.n_max_iterations) ? 103 : 0;  // 103: did not converge
            }
        }
        cudaMemcpyAsync(b->d_upd, upd.data(), np, cudaMemcpyHostToDevice, st);
        update_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_upd, b->d_mdu, b->d_u, b->d_ddu);
        if (b->npres > 0)
            update_multipliers_kernel<<<grid_of(b->npres), 256, 0, st>>>(b->npres, b->d_pres_prob, b->d_upd, b->d_mdl,
                                                                          b->d_lam);
        b->launches += 12;
    }
    b->launches += 4;
    if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "tick failed");
    return PMS_OK;
}

int pms_batch_solve_step(pms_batch* b, const double* c_values, const uint8_t* active, int32_t* iterations,
                         double* norm_rr, int32_t* status, int32_t* pcg_iterations) {
    if (!b || !active) return PMS_ERR_INVALID;
    const int np = b->np;
    std::vector<uint8_t> cmd(np, 0);
    std::vector<int32_t> res(np, -1), iter(np, 0), pcg(np, 0), pcg_sum(np, 0), stat(np, 0), count(np, 0);
    std::vector<double> norm(np, 0.0), last_norm(np, 0.0);
    for (int p = 0; p < np; p++) cmd[p] = active[p] ? 1 : 0;
    for (;;) {
        bool any = false;
        for (int p = 0; p < np; p++) any = any || cmd[p];
        if (!any) break;
        std::fill(pcg.begin(), pcg.end(), 0);
        int rc = pms_batch_tick(b, cmd.data(), c_values, res.data(), iter.data(), norm.data(), pcg.data());
        if (rc) return rc;
        for (int p = 0; p < np; p++) {
            if (!cmd[p]) continue;
            count[p] += 1;  // residual evaluations, as the reference counts iterations
            pcg_sum[p] += pcg[p];
            last_norm[p] = norm[p];
            if (res[p] == 0) {
                cmd[p] = 2;
            } else {
                cmd[p] = 0;
                stat[p] = (res[p] >= 100) ? res[p] - 100 : 0;
            }
        }
    }
    for (int p = 0; p < np; p++) {
        if (iterations) iterations[p] = count[p];
        if (norm_rr) norm_rr[p] = last_norm[p];
        if (status) status[p] = stat[p];
        if (pcg_iterations) pcg_iterations[p] = pcg_sum[p];
    }
    return PMS_OK;
}

int pms_batch_get_u(pms_batch* b, double* u) {
    if (!b || !u) return PMS_ERR_INVALID;
    if (cudaStreamSynchronize(b->v.stream) != cudaSuccess) return PMS_ERR_CUDA;
    return cudaMemcpy(u, b->d_u, b->ndof * 8, cudaMemcpyDeviceToHost) == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}

int pms_batch_get_multipliers(pms_batch* b, double* lam) {
    if (!b || !lam) return PMS_ERR_INVALID;
    if (cudaStreamSynchronize(b->v.stream) != cudaSuccess) return PMS_ERR_CUDA;
    if (b->npres == 0) return PMS_OK;
    return cudaMemcpy(lam, b->d_lam, b->npres * 8, cudaMemcpyDeviceToHost) == cudaSuccess ? PMS_OK : PMS_ERR_CUDA;
}

int64_t pms_batch_counters(const pms_batch* b, int64_t* pcg_iterations_total) {
    if (!b) return 0;
    if (pcg_iterations_total) *pcg_iterations_total = b->pcg_total;
    return b->launches;
}

const char* pms_batch_last_error(const pms_batch* b) { return b ? b->last_error.c_str() : "null handle"; }

}  // extern "C"
