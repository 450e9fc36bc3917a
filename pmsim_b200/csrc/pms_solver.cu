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
// Continuous progress.  A tick advances every running problem by one stage of its own Newton
// iteration: problems waiting for an element pass get it (all of them in one launch), problems
// whose linear solve is under way get up to `pcg_budget` more PCG iterations, and problems whose
// PCG converged in this tick finish their Newton iteration (multipliers, rel(mdu), U update).  A
// problem never waits for the PCG of another problem to finish.
//
// Two PCG engines, one arithmetic.  A problem whose vectors fit the shared memory of up to 16 CTAs
// runs its whole PCG loop on a thread-block cluster (pcg_team_kernel: distributed shared memory,
// hardware cluster barriers, every problem at its own pace, resumable across ticks); larger
// problems run the batch-wide kernels (spmv+dot, update, beta+direction), captured in a CUDA graph.  Both engines call the same per-node and per-row functions and reduce
// through the same trees: 128-node chunks that never straddle two problems, each summed by the
// fixed pairing (t, t+s), s = 64..1, and a problem's chunk partials summed in chunk order.  A
// problem's iterates are therefore bit-identical whichever engine runs it and whichever problems
// share the batch, so the engine threshold and launch shapes (chosen by pms_batch_autotune) change
// speed only.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pms.h"
#include "pms_device.cuh"
#include "pms_internal.h"

using namespace pms;

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int CHN = 128;        // nodes per reduction chunk (= threads per block of the node kernels)

struct SolverArgs {
    int nd;
    int np;
    int64_t nnode, ndof;
    const int32_t* node_prob;    // problem of each node
    const int64_t* chunk_node0;  // first node of each chunk
    const int32_t* chunk_nnode;  // nodes in each chunk
    const int32_t* chunk_prob;   // problem of each chunk
    const int64_t* pchunk;       // chunks of problem p: [pchunk[p], pchunk[p+1])
    const int32_t* pres_idx;     // per DOF: index into the prescribed arrays, or -1
    const uint8_t* active;       // per problem: selected for the current Newton-level stage
    uint8_t* pcg_active;         // [2][np]: PCG still iterating on the batch-wide engine (by parity)
    const uint8_t* engine;       // per problem: 1 = block engine, 0 = batch-wide engine
};

// ---- canonical reductions ----------------------------------------------------------------
// A 128-node chunk is summed as four 32-node quarters, each by the warp shuffle tree (pairs t, t+16,
// t+8, ..., t+1), and the quarters as ((q0 + q1) + (q2 + q3)).  Every block-level PCG and Newton
// reduction goes through here (threads [128g, 128g + 128) of a block form group g and hold the
// chunk's nodes in order), and a kernel that gives each quarter its own block reproduces the same
// value; so a problem's dot products do not depend on the engine that computes them.
template <bool MAX>
__device__ __forceinline__ double warp_tree(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_down_sync(FULL, v, o);
        v = MAX ? fmax(v, w) : v + w;
    }
    return v;  // lane 0 holds the quarter's value
}

template <bool MAX>
__device__ __forceinline__ double quarters(double q0, double q1, double q2, double q3) {
    return MAX ? fmax(fmax(q0, q1), fmax(q2, q3)) : (q0 + q1) + (q2 + q3);
}

// All threads of the block must call it; sh holds at least 4 doubles per group.  trailing = false
// leaves out the barrier that protects sh from the block's next write to it: for a caller whose next
// write to sh follows another block (or cluster) barrier anyway, or goes to another region.
template <bool MAX>
__device__ __forceinline__ double group_reduce(double v, double* sh, bool trailing = true) {
    const double w = warp_tree<MAX>(v);
    double* s = sh + 4 * (threadIdx.x / CHN);
    if ((threadIdx.x & 31) == 0) s[(threadIdx.x & (CHN - 1)) >> 5] = w;
    __syncthreads();
    const double r = quarters<MAX>(s[0], s[1], s[2], s[3]);
    if (trailing) __syncthreads();
    return r;
}

// Two sums at once (same trees as two group_reduce<false> calls); sh holds 8 doubles per group.
__device__ __forceinline__ void group_reduce2(double& a, double& b, double* sh, bool trailing = true) {
    const double wa = warp_tree<false>(a), wb = warp_tree<false>(b);
    double* s = sh + 8 * (threadIdx.x / CHN);
    if ((threadIdx.x & 31) == 0) {
        const int k = (threadIdx.x & (CHN - 1)) >> 5;
        s[k] = wa;
        s[4 + k] = wb;
    }
    __syncthreads();
    a = quarters<false>(s[0], s[1], s[2], s[3]);
    b = quarters<false>(s[4], s[5], s[6], s[7]);
    if (trailing) __syncthreads();
}

// Total of a problem's chunk partials (the per-problem half of every PCG reduction), computed by a
// group of 128 threads: thread t adds the partials t, t+128, ... in order, then the group tree.
// Every PCG engine computes its totals this way, so they agree to the bit.
__device__ __forceinline__ double problem_total(const double* part, int64_t c0, int64_t c1, double* sh,
                                                bool trailing = true) {
    double s = 0.0;
    for (int64_t c = c0 + (threadIdx.x & (CHN - 1)); c < c1; c += CHN) s += part[c];
    return group_reduce<false>(s, sh, trailing);
}

// The same total from quarter partials (four per chunk, in chunk order).
__device__ __forceinline__ double problem_total_quarters(const double* part4, int64_t c0, int64_t c1, double* sh) {
    double s = 0.0;
    for (int64_t c = c0 + (threadIdx.x & (CHN - 1)); c < c1; c += CHN)
        s += quarters<false>(part4[4 * c], part4[4 * c + 1], part4[4 * c + 2], part4[4 * c + 3]);
    return group_reduce<false>(s, sh);
}

__device__ __forceinline__ void problem_total2(const double* pa, const double* pb, int64_t c0, int64_t c1,
                                               double& a, double& b, double* sh, bool trailing = true) {
    a = 0.0;
    b = 0.0;
    for (int64_t c = c0 + (threadIdx.x & (CHN - 1)); c < c1; c += CHN) {
        a += pa[c];
        b += pb[c];
    }
    group_reduce2(a, b, sh, trailing);
}

// ---- per-row / per-node PCG arithmetic shared by both engines -----------------------------
// (K x)_row by TPR lanes: lane `sub` takes the entries sub, sub+TPR, ... (FMA chain), then a
// shuffle tree over the TPR lanes.  Every lane of the warp must call it (on = false: no entries).
template <int TPR>
__device__ __forceinline__ double row_dot(int64_t row, int sub, bool on, const int64_t* __restrict__ indptr,
                                          const int32_t* __restrict__ indices, const double* __restrict__ val,
                                          const double* __restrict__ x) {
    double s = 0.0;
    if (on)
        for (int64_t k = indptr[row] + sub; k < indptr[row + 1]; k += TPR) s = fma(val[k], x[indices[k]], s);
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o, TPR);
    return s;
}

// The ND rows of node A of K in the node-block layout of the element handle: block row A holds nba
// ND x ND blocks from bb = bptr[A], row i of the node at val[ND*ND*bb + i*ND*nba + pos*ND + j], block
// columns bcol[bb + pos].  TPR lanes: lane sub takes the blocks pos = sub, sub + TPR, ... two per round
// (both loaded before either is added), each block's FMAs in (i, j) order, then a shuffle tree per row.
// Every lane of the warp calls it (nba = 0 for a lane group without a node); gather(B, x) supplies
// x[B*ND + 0 .. ND-1].  The PCG engines all use it, so their iterates agree bit for bit.
template <int ND, int TPR, class GatherN>
__device__ __forceinline__ void node_rows_dot(int64_t bb, int nba, int sub, const double* __restrict__ val,
                                              const int32_t* __restrict__ bcol, const GatherN& gather,
                                              double (&s)[ND]) {
#pragma unroll
    for (int i = 0; i < ND; i++) s[i] = 0.0;
    const double* v = val + (int64_t)ND * ND * bb;
    const int rs = ND * nba;
    for (int pos = sub; pos < nba; pos += 2 * TPR) {
        const int p1 = pos + TPR;
        const bool two = p1 < nba;
        const int32_t c0 = bcol[bb + pos];
        const int32_t c1 = two ? bcol[bb + p1] : c0;
        double a0[ND][ND], a1[ND][ND], x0[ND], x1[ND];
#pragma unroll
        for (int i = 0; i < ND; i++)
#pragma unroll
            for (int j = 0; j < ND; j++) {
                a0[i][j] = v[i * rs + pos * ND + j];
                a1[i][j] = two ? v[i * rs + p1 * ND + j] : 0.0;
            }
        gather(c0, x0);
        gather(c1, x1);
#pragma unroll
        for (int i = 0; i < ND; i++)
#pragma unroll
            for (int j = 0; j < ND; j++) s[i] = fma(a0[i][j], x0[j], s[i]);
        if (two) {
#pragma unroll
            for (int i = 0; i < ND; i++)
#pragma unroll
                for (int j = 0; j < ND; j++) s[i] = fma(a1[i][j], x1[j], s[i]);
        }
    }
#pragma unroll
    for (int i = 0; i < ND; i++)
#pragma unroll
        for (int o = TPR / 2; o > 0; o >>= 1) s[i] += __shfl_down_sync(FULL, s[i], o, TPR);
}

// a.b over the free DOFs of a node; pres, a, b point at the node's first DOF
template <class P>
__device__ __forceinline__ double node_dot(const P* pres, int nd, const double* a, const double* b) {
    double s = 0.0;
    for (int d = 0; d < nd; d++)
        if (pres[d] < 0) s = fma(a[d], b[d], s);
    return s;
}

// x += alpha p, r -= alpha q (free DOFs), z = M r with the node's inverse diagonal block B;
// accumulates the node's r.z and r.r (all pointers at the node's first DOF / block)
template <class P>
__device__ __forceinline__ void node_update(const P* pres, int nd, double alpha, const double* p,
                                            const double* q, const double* B, double* x, double* r, double* z,
                                            double& rz, double& r2) {
    double rv[3];
    for (int d = 0; d < nd; d++) {
        if (pres[d] < 0) {
            x[d] = fma(alpha, p[d], x[d]);
            rv[d] = fma(-alpha, q[d], r[d]);
            r[d] = rv[d];
        } else {
            rv[d] = 0.0;
        }
    }
    for (int d = 0; d < nd; d++) {
        double zv = 0.0;
        for (int e = 0; e < nd; e++) zv = fma(B[d * nd + e], rv[e], zv);
        z[d] = zv;
        rz = fma(rv[d], zv, rz);
        r2 = fma(rv[d], rv[d], r2);
    }
}

// p = z + beta p on a DOF (0 on prescribed DOFs)
template <class P>
__device__ __forceinline__ void dof_direction(P pres, double beta, const double* z, double* p) {
    *p = (pres >= 0) ? 0.0 : fma(beta, *p, *z);
}

// scalar step of one PCG iteration: beta, rho, iteration count and the stopping test
__device__ __forceinline__ bool pcg_scalar_step(double rz, double rr, double& rho, double r0, int32_t& iters,
                                                double rtol, int32_t max_iter, double& beta) {
    beta = (rho != 0.0) ? rz / rho : 0.0;
    rho = rz;
    iters += 1;
    return !(sqrt(rr) > rtol * r0) || iters >= max_iter;  // true: done
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
    m = group_reduce<true>(m, sh);
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
    const bool ok = spd_block_inverse(a, nf);
    double* out = binv + node * nd * nd;
    for (int i = 0; i < nd * nd; i++) out[i] = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) out[fr[i] * nd + fr[j]] = ok ? a[i][nf + j] : (i == j ? 1.0 / fmax(fabs(a[i][i]), 1e-300) : 0.0);
}

// y = K x on the rows of the problems with flag[p] set (TPR threads per row); y_p = 0 on
// prescribed rows when mask_pres.
template <int TPR>
__global__ void spmv_kernel(SolverArgs S, const int64_t* indptr, const int32_t* indices, const double* val,
                            const double* x, double* y, const uint8_t* flag, bool mask_pres) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t row = gid / TPR;
    const int sub = (int)(gid % TPR);
    // no early exit: every lane of the warp takes part in the shuffles
    const bool on = row < S.ndof && flag[S.node_prob[row < S.ndof ? row / S.nd : 0]];
    const double s = row_dot<TPR>(row, sub, on, indptr, indices, val, x);
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
    __shared__ double sh[2 * CHN];
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
            for (int e = 0; e < nd; e++) zv = fma(B[d * nd + e], rv[e], zv);
            z[node * nd + d] = zv;
            p[node * nd + d] = zv;
            rz = fma(rv[d], zv, rz);
            r2 = fma(rv[d], rv[d], r2);
        }
    }
    group_reduce2(rz, r2, sh);
    if (threadIdx.x == 0 && S.active[pr]) {
        part_rz[ch] = rz;
        part_rr[ch] = r2;
    }
}

// per problem selected by `active` (one block of 128 threads each): rho = r.z, r0 = |r|_2, iteration
// count 0, and the engine that runs its PCG (block engine: cta_active, batch-wide: pcg_active)
__global__ void __launch_bounds__(CHN)
pcg_init_scalars_kernel(int np, const uint8_t* active, const uint8_t* engine, const int64_t* pchunk,
                        const double* part_rz, const double* part_rr, double* rho, double* r0, uint8_t* pcg_active,
                        uint8_t* cta_active, int32_t* pcg_iters) {
    __shared__ double sh[2 * CHN];
    const int p = blockIdx.x;
    if (!active[p]) return;
    double a, b;
    problem_total2(part_rz, part_rr, pchunk[p], pchunk[p + 1], a, b, sh);
    if (threadIdx.x != 0) return;
    r0[p] = sqrt(b);
    const uint8_t go = b > 0.0 ? 1 : 0;
    for (int e = 0; e < 2; e++) {  // both parity buffers of the batch-wide engine
        rho[e * np + p] = a;
        pcg_active[e * np + p] = engine[p] ? 0 : go;
        pcg_iters[e * np + p] = 0;
    }
    cta_active[p] = engine[p] ? go : 0;
}

// ---- batch-wide PCG engine (one CUDA graph node per kernel) --------------------------------

// q = K p on the nodes of one chunk quarter (32 nodes, one group of TPR lanes each, node_rows_dot),
// then the quarter's partial of p.q by the warp tree.  Block b covers quarter b % 4 of chunk b / 4.
template <int TPR>
__host__ __device__ constexpr int quarter_threads() { return 32 * TPR; }

template <int TPR>
__global__ void __launch_bounds__(quarter_threads<TPR>())
pcg_spmv_dot_kernel(SolverArgs S, int par, const int64_t* __restrict__ bptr, const int32_t* __restrict__ bcol,
                    const double* __restrict__ val, const double* p, double* q, double* part4) {
    constexpr int ND = TPR == 8 ? 2 : 3;  // the lanes per node follow the dimension
    const int64_t ch = blockIdx.x >> 2;
    const int k = blockIdx.x & 3;
    const int pr = S.chunk_prob[ch];
    if (!S.pcg_active[par * S.np + pr]) return;  // whole block
    const int nn = max(0, min(32, S.chunk_nnode[ch] - 32 * k));
    const int64_t node0 = S.chunk_node0[ch] + 32 * k;
    const int grp = threadIdx.x / TPR, sub = threadIdx.x % TPR;
    const bool on = grp < nn;
    const int64_t A = node0 + grp;
    const int64_t bb = on ? bptr[A] : 0;
    const int nba = on ? (int)(bptr[A + 1] - bb) : 0;
    double sv[ND];
    node_rows_dot<ND, TPR>(bb, nba, sub, val, bcol,
                           [&](int32_t c, double (&x)[ND]) {
#pragma unroll
                               for (int j = 0; j < ND; j++) x[j] = p[(int64_t)c * ND + j];
                           },
                           sv);
    if (on && sub == 0) {
#pragma unroll
        for (int i = 0; i < ND; i++) q[A * ND + i] = (S.pres_idx[A * ND + i] >= 0) ? 0.0 : sv[i];
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int64_t i0 = (node0 + threadIdx.x) * S.nd;
        const double v = (threadIdx.x < nn) ? node_dot(S.pres_idx + i0, S.nd, p + i0, q + i0) : 0.0;
        const double t = warp_tree<false>(v);
        if (threadIdx.x == 0) part4[4 * ch + k] = t;
    }
}

// alpha = rho / p.q (every block of a problem sums the same partials in the same order), then
// x, r, z and the chunk's partials of r.z and r.r
__global__ void __launch_bounds__(CHN)
pcg_update_kernel(SolverArgs S, int par, const double* part_pq /*4 per chunk*/, const double* rho, const double* p,
                  const double* q,
                  const double* binv, double* x, double* r, double* z, double* part_rz, double* part_rr,
                  int32_t* nactive) {
    __shared__ double sh[2 * CHN];
    if (blockIdx.x == 0 && threadIdx.x == 0) *nactive = 0;  // counted again by pcg_beta_direction_kernel
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    if (!S.pcg_active[par * S.np + pr]) return;  // whole block
    const double pq = problem_total_quarters(part_pq, S.pchunk[pr], S.pchunk[pr + 1], sh);
    const double alpha = (pq != 0.0) ? rho[par * S.np + pr] / pq : 0.0;
    double rz = 0.0, r2 = 0.0;
    if (threadIdx.x < S.chunk_nnode[ch]) {
        const int nd = S.nd;
        const int64_t node = S.chunk_node0[ch] + threadIdx.x, i0 = node * nd;
        node_update(S.pres_idx + i0, nd, alpha, p + i0, q + i0, binv + node * nd * nd, x + i0, r + i0, z + i0, rz, r2);
    }
    group_reduce2(rz, r2, sh);
    if (threadIdx.x == 0) {
        part_rz[ch] = rz;
        part_rr[ch] = r2;
    }
}

// beta (every block of a problem from the same partials), the direction p = z + beta p on the
// chunk, and -- by the problem's first chunk -- rho, the iteration count and the stopping test.
// The per-problem scalars are double-buffered by iteration parity (read `par`, write the other),
// so no block reads a value that another block of the same launch writes; graphs hold an even
// number of iterations, so buffer 0 is current between launches.
__global__ void __launch_bounds__(CHN)
pcg_beta_direction_kernel(SolverArgs S, int par, const double* part_rz, const double* part_rr, double* rho,
                          const double* r0, double rtol, int32_t max_iter, int32_t* iters, const double* z, double* p,
                          int32_t* nactive) {
    __shared__ double sh[2 * CHN];
    const int64_t ch = blockIdx.x;
    const int pr = S.chunk_prob[ch];
    if (S.engine[pr]) return;  // block-engine problem: its state is not ours
    const int cur = par * S.np + pr, nxt = (par ^ 1) * S.np + pr;
    const bool lead = ch == S.pchunk[pr];
    if (!S.pcg_active[cur]) {
        if (lead && threadIdx.x == 0) {
            S.pcg_active[nxt] = 0;
            rho[nxt] = rho[cur];
            iters[nxt] = iters[cur];
        }
        return;
    }
    double a, b;
    problem_total2(part_rz, part_rr, S.pchunk[pr], S.pchunk[pr + 1], a, b, sh);
    double rh = rho[cur], beta;
    int32_t it = iters[cur];
    const bool done = pcg_scalar_step(a, b, rh, r0[pr], it, rtol, max_iter, beta);
    if (lead && threadIdx.x == 0) {
        rho[nxt] = rh;
        iters[nxt] = it;
        S.pcg_active[nxt] = done ? 0 : 1;
        if (!done) atomicAdd(nactive, 1);
    }
    if (threadIdx.x < S.chunk_nnode[ch]) {
        const int64_t node = S.chunk_node0[ch] + threadIdx.x;
        for (int d = 0; d < S.nd; d++) {
            const int64_t i = node * S.nd + d;
            dof_direction(S.pres_idx[i], beta, z + i, p + i);
        }
    }
}

// ---- team PCG engine: a thread-block cluster runs one problem's PCG --------------------------
// Problem list[blockIdx.x / C] runs on the C CTAs of one cluster (C = 1..16).  CTA k owns a
// contiguous run of the problem's 128-node chunks and keeps x, r, z, p, q and the preconditioner of
// its nodes in shared memory; the SpMV reads the p of nodes owned by other CTAs of the cluster
// through distributed shared memory.  Chunk partials are stored into every CTA's copy of the
// partial arrays, so that each CTA forms the same problem totals.  Hardware cluster barriers order
// the phases (no spin waits).  Up to `budget` iterations (or to convergence) per launch; the state
// goes back to global memory at the end, so the next launch resumes.  Same arithmetic as the
// batch-wide kernels: bit-identical iterates.
constexpr int TEAM_MAX = 16;
constexpr int TEAM_MAX_CHUNKS = 256;  // chunks of a team problem
constexpr size_t TEAM_SMEM_LIMIT = 200 * 1024;

// Shared memory of a team CTA: doubles p, q, r, z, x (npc*nd each), the inverse diagonal blocks
// (npc*nd*nd), three chunk-partial arrays and the reduction scratch (2*bd); then int32 block
// pointers of its nodes (npc*nd + 1 room) and the CTAs' node offsets (TEAM_MAX + 1); then one byte
// per DOF (-1 free, 0 prescribed).
__host__ __device__ inline size_t team_fixed_bytes(int bd) {
    return (size_t)8 * (3 * TEAM_MAX_CHUNKS + 2 * bd) + 4 * (TEAM_MAX + 2) + 16;
}
__host__ __device__ inline size_t team_node_bytes(int nd) { return (size_t)8 * (5 * nd + nd * nd) + 5 * nd; }
// nodes per CTA a team kernel can hold (a multiple of the chunk size)
__host__ __device__ inline int team_node_capacity(int nd, int bd) {
    const int nodes = (int)((TEAM_SMEM_LIMIT - team_fixed_bytes(bd)) / team_node_bytes(nd));
    return (nodes / CHN) * CHN;
}
__host__ __device__ inline size_t team_smem_bytes(int nd, int bd) {
    return team_fixed_bytes(bd) + (size_t)team_node_capacity(nd, bd) * team_node_bytes(nd);
}

template <int BD, int TPR>
__global__ void __launch_bounds__(BD, 1)
pcg_team_kernel(SolverArgs S, const int32_t* list, const int64_t* __restrict__ bptr,
                const int32_t* __restrict__ bcol, const double* __restrict__ val, const double* binv_g,
                double* x_g, double* r_g, double* z_g, double* p_g, double* rho_g, const double* r0_g,
                int32_t* iters_g, uint8_t* cta_active, double rtol, int32_t max_iter, int32_t budget) {
    namespace cg = cooperative_groups;
    constexpr int G = BD / CHN;
    constexpr int nd = TPR == 8 ? 2 : 3;    // DOFs per node (the lanes per node follow the dimension)
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int me = (int)cl.block_rank();
    const int pr = list[blockIdx.x / C];
    if (!cta_active[pr]) return;  // the whole cluster reads the same flag
    // a one-CTA team needs no cluster barrier (its partials are its own shared memory)
    auto team_sync = [&]() {
        if (C == 1) __syncthreads();
        else cl.sync();
    };
    const int npc = team_node_capacity(nd, BD);
    extern __shared__ double smem[];
    double* ps = smem;
    double* qs = ps + npc * nd;
    double* rs = qs + npc * nd;
    double* zs = rs + npc * nd;
    double* xs = zs + npc * nd;
    double* bs = xs + npc * nd;                  // npc * nd * nd
    double* part_pq = bs + npc * nd * nd;        // TEAM_MAX_CHUNKS each
    double* part_rz = part_pq + TEAM_MAX_CHUNKS;
    double* part_rr = part_rz + TEAM_MAX_CHUNKS;
    double* red = part_rr + TEAM_MAX_CHUNKS;     // 2 * BD
    int32_t* rp = (int32_t*)(red + 2 * BD);      // block pointers of my nodes (relative; npc * nd + 1 room)
    int32_t* kb = rp + npc * nd + 1;             // TEAM_MAX + 1 node offsets of the CTAs' runs
    int8_t* fr = (int8_t*)(kb + TEAM_MAX + 1);   // npc * nd: -1 free DOF, 0 prescribed
    const int64_t c0 = S.pchunk[pr];
    const int nch = (int)(S.pchunk[pr + 1] - c0);
    const int64_t n0 = S.chunk_node0[c0];
    const int N = (int)(S.chunk_node0[c0 + nch - 1] + S.chunk_nnode[c0 + nch - 1] - n0);  // nodes
    if (threadIdx.x <= C) {
        const int k = (int)threadIdx.x;
        kb[k] = min(N, CHN * (int)((int64_t)k * nch / C));
    }
    __syncthreads();
    const int cb = (int)((int64_t)me * nch / C), ce = (int)((int64_t)(me + 1) * nch / C);  // my chunks
    const int nb = kb[me], ne = kb[me + 1];                                               // my nodes
    const int64_t gd0 = (n0 + nb) * nd;  // my first DOF (= first row)
    const int nloc = ne - nb, ndl = nloc * nd;
    const int64_t bbase = bptr[n0 + nb];
    for (int i = threadIdx.x; i < ndl; i += BD) {
        ps[i] = p_g[gd0 + i];
        rs[i] = r_g[gd0 + i];
        zs[i] = z_g[gd0 + i];
        xs[i] = x_g[gd0 + i];
        fr[i] = S.pres_idx[gd0 + i] < 0 ? -1 : 0;
    }
    for (int i = threadIdx.x; i <= nloc; i += BD) rp[i] = (int32_t)(bptr[n0 + nb + i] - bbase);
    for (int i = threadIdx.x; i < ndl * nd; i += BD) bs[i] = binv_g[gd0 * nd + i];
    double rho = rho_g[pr];
    const double r0 = r0_g[pr];
    int32_t it = iters_g[pr];
    bool active = true;
    const int g = threadIdx.x / CHN, tg = threadIdx.x % CHN;
    const int sub = threadIdx.x % TPR, grp = threadIdx.x / TPR;
    // p of node B of the problem: from my shared memory or from the owning CTA's
    auto gather = [&](int32_t B, double (&xv)[nd]) {
        const int node = B - (int)n0;
        const double* src;
        if (node >= nb && node < ne) {
            src = ps + (node - nb) * nd;
        } else {
            // owner of chunk c: the largest k with floor(k*nch/C) <= c
            const int k = (int)(((int64_t)(node / CHN + 1) * C - 1) / nch);
            src = cl.map_shared_rank(ps, k) + (node - kb[k]) * nd;
        }
#pragma unroll
        for (int j = 0; j < nd; j++) xv[j] = src[j];
    };
    team_sync();  // every CTA holds its p before the first remote read
    for (int step = 0; step < budget && active; step++) {
        // q = K p on my nodes (one group of TPR lanes per node)
        for (int base = 0; base < nloc; base += BD / TPR) {
            const int ln = base + grp;
            const bool on = ln < nloc;
            const int64_t bb = on ? bbase + rp[ln] : 0;
            const int nba = on ? rp[ln + 1] - rp[ln] : 0;
            double sv[nd];
            node_rows_dot<nd, TPR>(bb, nba, sub, val, bcol, gather, sv);
            if (on && sub == 0) {
#pragma unroll
                for (int i = 0; i < nd; i++) qs[ln * nd + i] = (fr[ln * nd + i] >= 0) ? 0.0 : sv[i];
            }
        }
        __syncthreads();
        // p.q partials of my chunks, stored into every CTA's array
        for (int j0 = cb; j0 < ce; j0 += G) {
            const int j = j0 + g;
            double v = 0.0;
            if (j < ce && tg < min(CHN, N - CHN * j)) {
                const int l = (CHN * j - nb + tg) * nd;
                v = node_dot(fr + l, nd, ps + l, qs + l);
            }
            v = group_reduce<false>(v, red, j0 + G < ce);  // (region A; the cluster barrier follows)
            if (tg == 0 && j < ce)
                for (int k = 0; k < C; k++) cl.map_shared_rank(part_pq, k)[j] = v;
        }
        team_sync();
        const double pq = problem_total(part_pq, 0, nch, red + 8 * G, false);  // region B: nothing else writes it
        const double alpha = (pq != 0.0) ? rho / pq : 0.0;
        for (int j0 = cb; j0 < ce; j0 += G) {
            const int j = j0 + g;
            double rz = 0.0, r2 = 0.0;
            if (j < ce && tg < min(CHN, N - CHN * j)) {
                const int ln = CHN * j - nb + tg, l = ln * nd;
                node_update(fr + l, nd, alpha, ps + l, qs + l, bs + ln * nd * nd, xs + l, rs + l, zs + l, rz, r2);
            }
            group_reduce2(rz, r2, red + 16 * G, j0 + G < ce);  // region C; the cluster barrier follows
            if (tg == 0 && j < ce)
                for (int k = 0; k < C; k++) {
                    cl.map_shared_rank(part_rz, k)[j] = rz;
                    cl.map_shared_rank(part_rr, k)[j] = r2;
                }
        }
        team_sync();
        double rzt, rrt, beta;
        problem_total2(part_rz, part_rr, 0, nch, rzt, rrt, red, false);  // region A, last written before two barriers
        const bool done = pcg_scalar_step(rzt, rrt, rho, r0, it, rtol, max_iter, beta);
        for (int i = threadIdx.x; i < ndl; i += BD) dof_direction(fr[i], beta, zs + i, ps + i);
        active = !done;
        team_sync();  // p complete (and every remote read of this iteration done) before the next SpMV
    }
    for (int i = threadIdx.x; i < ndl; i += BD) {
        p_g[gd0 + i] = ps[i];
        r_g[gd0 + i] = rs[i];
        z_g[gd0 + i] = zs[i];
        x_g[gd0 + i] = xs[i];
    }
    if (me == 0 && threadIdx.x == 0) {
        rho_g[pr] = rho;
        iters_g[pr] = it;
        cta_active[pr] = active ? 1 : 0;
    }
    team_sync();  // no CTA leaves while another may still address its shared memory
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
    m = group_reduce<true>(m, sh);
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

__global__ void fill_masked_kernel(SolverArgs S, const uint8_t* flag, double* v, double value) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S.ndof) return;
    if (flag[S.node_prob[i / S.nd]]) v[i] = value;
}

// ---- device-resident load step (pms_batch_solve_step_graph) --------------------------------
// One CUDA graph per load step: a conditional WHILE over Newton iterations, each one the element pass,
// the residual test, the PCG start, a nested WHILE over PCG iterations (batch-wide engine), the
// completion and the update.  The per-problem sequencing of pms_batch_tick (and of
// SolverImplicit::iterate, src/fem/solver_implicit.rs:187-272) runs in these controller kernels
// instead of on the host; each problem's arithmetic is the same kernels' and gives the same bits.
enum : uint8_t { PH_IDLE = 0, PH_START = 1, PH_CONT = 2, PH_SOLVE = 3 };

__global__ void step_init_kernel(int np, const uint8_t* sel, uint8_t* phase, int32_t* st, int32_t* cnt,
                                 int32_t* pcgsum, double* lastnorm) {
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        phase[p] = sel[p] ? PH_START : PH_IDLE;
        st[p] = 0;
        cnt[p] = 0;
        pcgsum[p] = 0;
        lastnorm[p] = 0.0;
    }
}

// element modes of this iteration (1: new step, 2: continue), dU = 0 mask of the new steps
__global__ void step_pre_elem_kernel(int np, const uint8_t* phase, uint8_t* pmode, uint8_t* start, uint8_t* active,
                                     int32_t* it, unsigned long long* perr, int constant_tangent) {
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const uint8_t ph = phase[p];
        const uint8_t m = ph == PH_START ? 1 : (ph == PH_CONT ? (constant_tangent ? 3 : 2) : 0);
        pmode[p] = m;
        start[p] = ph == PH_START;
        active[p] = m != 0;
        if (ph == PH_START) it[p] = 0;
        perr[p] = 0;
    }
}

// after the residual: element errors, NaN/Inf, convergence on max|R|, or on to the linear solve
__global__ void step_post_resid_kernel(int np, cudaGraphConditionalHandle pcg_loop, double tol_rr,
                                       const unsigned long long* perr, const double* norm, uint8_t* phase,
                                       uint8_t* active, uint8_t* first, const int32_t* it, int32_t* st, int32_t* cnt,
                                       double* lastnorm) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        if (!active[p]) continue;
        cnt[p] += 1;  // a residual evaluation, as the reference counts iterations
        const int code = (int)(perr[p] & 0xff);
        uint8_t solve = 0;
        if (perr[p] != 0 && (code == 3 || code == 4 || code == 5)) {
            st[p] = 101 + code;  // 104 zero sigma_d, 105 zero norm_s, 106 Jacobian
            phase[p] = PH_IDLE;
        } else {
            lastnorm[p] = norm[p];
            if (!isfinite(norm[p])) {
                st[p] = 101;  // "Found NaN or Inf"
                phase[p] = PH_IDLE;
            } else if (norm[p] < tol_rr) {
                st[p] = 1;
                phase[p] = PH_IDLE;
            } else {
                solve = 1;
                phase[p] = PH_SOLVE;
                first[p] = it[p] == 0;
                any = 1;
            }
        }
        active[p] = solve;
    }
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(pcg_loop, any ? 1u : 0u);
}

__global__ void step_cond_pcg_kernel(cudaGraphConditionalHandle pcg_loop, const int32_t* nactive) {
    cudaGraphSetConditional(pcg_loop, *nactive > 0 ? 1u : 0u);
}

// after the linear solve: NaN/Inf in mdu, convergence on rel(mdu) (not applied), or the update
__global__ void step_post_complete_kernel(int np, int max_it, double tol_mdu, const double* rel, const uint8_t* active,
                                          const int32_t* pcg_iters, uint8_t* phase, uint8_t* upd, int32_t* it,
                                          int32_t* st, int32_t* pcgsum) {
    for (int p = threadIdx.x; p < np; p += blockDim.x) {
        upd[p] = 0;
        if (!active[p]) continue;
        pcgsum[p] += pcg_iters[p];  // parity buffer 0: the PCG loop runs an even number of iterations
        if (!isfinite(rel[p])) {
            st[p] = 102;  // "Found NaN or Inf in mdu"
            phase[p] = PH_IDLE;
        } else if (it[p] > 0 && rel[p] < tol_mdu) {
            st[p] = 1;
            phase[p] = PH_IDLE;
        } else {
            upd[p] = 1;
            it[p] += 1;
            if (it[p] >= max_it) {
                st[p] = 103;  // "Newton-Raphson did not converge" (the update is applied, as in the tick)
                phase[p] = PH_IDLE;
            } else {
                phase[p] = PH_CONT;
            }
        }
    }
}

__global__ void step_cond_newton_kernel(int np, cudaGraphConditionalHandle newton_loop, const uint8_t* phase) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int p = threadIdx.x; p < np; p += blockDim.x)
        if (phase[p] == PH_START || phase[p] == PH_CONT) any = 1;
    __syncthreads();
    if (threadIdx.x == 0) cudaGraphSetConditional(newton_loop, any ? 1u : 0u);
}

}  // namespace

// ------------------------------------------------------------------------------------ handle
struct pms_batch {
    pms_elements* el = nullptr;
    ElementsView v{};
    int np = 0;
    int64_t nnode = 0, ndof = 0, npres = 0, nchunk = 0;
    pms_batch_config cfg{};
    pms_batch_tuning tune{};
    std::vector<int64_t> point_ptr, cell_ptr, pres_ptr;
    std::vector<void*> allocs;
    // device
    int32_t *d_node_prob = nullptr, *d_cell_prob = nullptr, *d_chunk_nnode = nullptr, *d_chunk_prob = nullptr;
    int64_t *d_chunk_node0 = nullptr, *d_pchunk = nullptr, *d_ppres = nullptr, *d_pres_eq = nullptr;
    int32_t *d_pres_idx = nullptr, *d_pres_prob = nullptr, *d_list = nullptr;
    uint8_t *d_active = nullptr, *d_pcg_active = nullptr, *d_cta_active = nullptr, *d_pmode = nullptr,
            *d_first = nullptr, *d_upd = nullptr, *d_engine = nullptr;
    double *d_u = nullptr, *d_ddu = nullptr, *d_ff = nullptr, *d_fext = nullptr, *d_csr = nullptr, *d_rr = nullptr;
    double *d_mdu = nullptr, *d_mdu0 = nullptr, *d_kt = nullptr, *d_r = nullptr, *d_z = nullptr, *d_p = nullptr,
           *d_q = nullptr, *d_x = nullptr, *d_binv = nullptr;
    double *d_lam = nullptr, *d_c = nullptr, *d_mdl = nullptr, *d_mdl0 = nullptr;
    double *d_part_a = nullptr, *d_part_b = nullptr, *d_part_c = nullptr;
    double *d_rho = nullptr, *d_r0 = nullptr, *d_norm = nullptr, *d_rel = nullptr;
    int32_t *d_iters = nullptr, *d_nactive = nullptr;
    int64_t* d_queue = nullptr;    // work queue of the element pass: 4 arrays of np + 1
    unsigned long long* d_perr = nullptr;  // per problem: key of its element error in the last pass
    // device-resident load step
    cudaGraphExec_t step_graph = nullptr;
    uint8_t *d_phase = nullptr, *d_sel = nullptr, *d_zero_engine = nullptr;
    int32_t *d_st = nullptr, *d_cnt = nullptr, *d_pcgsum = nullptr, *d_it = nullptr;
    double* d_lastnorm = nullptr;
    std::vector<int64_t> h_queue;
    const int64_t* d_indptr = nullptr;
    const int32_t* d_indices = nullptr;
    SolverArgs S{};
    cudaStream_t st_cls[5] = {};  // team launches (one stream per team size), beside the batch-wide engine
    cudaEvent_t ev_fork = nullptr, ev_cls[5] = {};
    int cls_off[6] = {};
    int team_cmax = 8;
    cudaGraphExec_t graph = nullptr;
    int graph_iters_captured = 0;
    std::string last_error;
    int64_t launches = 0;
    int64_t pcg_total = 0;
    int64_t host_syncs = 0;  // host waits for the device inside the Newton loop (instrumentation)
    std::vector<int32_t> it;       // Newton iteration of each problem within its current load step
    std::vector<uint8_t> solving;  // per problem: linear solve under way
    std::vector<uint8_t> engine;   // per problem: 1 = block engine, 0 = batch-wide engine
    std::vector<int64_t> pndof;    // DOFs of each problem
    std::vector<int64_t> pnch;     // reduction chunks of each problem
    std::vector<int32_t> h_list;

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
        for (auto c : st_cls)
            if (c) cudaStreamSynchronize(c);
        std::lock_guard<std::mutex> lock(device_mutex());
        if (graph) cudaGraphExecDestroy(graph);
        if (step_graph) cudaGraphExecDestroy(step_graph);
        if (ev_fork) cudaEventDestroy(ev_fork);
        for (auto e : ev_cls)
            if (e) cudaEventDestroy(e);
        for (auto c : st_cls)
            if (c) cudaStreamDestroy(c);
        for (void* p : allocs) cudaFree(p);
    }
};

namespace {

int bfail(pms_batch* b, int code, const char* msg) {
    if (b) b->last_error = msg;
    return code;
}

inline unsigned grid_of(int64_t n, int t = 256) { return (unsigned)std::max<int64_t>((n + t - 1) / t, 1); }

int tpr_of(int nd) { return nd == 2 ? 8 : 16; }

void launch_spmv(pms_batch* b, const double* x, double* y, const uint8_t* flag, bool mask) {
    const int tpr = tpr_of(b->v.nd);
    const int64_t threads = b->ndof * tpr;
    if (tpr == 8)
        spmv_kernel<8><<<grid_of(threads), 256, 0, b->v.stream>>>(b->S, b->d_indptr, b->d_indices, b->d_csr, x, y,
                                                                   flag, mask);
    else
        spmv_kernel<16><<<grid_of(threads), 256, 0, b->v.stream>>>(b->S, b->d_indptr, b->d_indices, b->d_csr, x, y,
                                                                    flag, mask);
    b->launches++;
}

// Appends a kernel node (after `dep`, if any) to graph g; args point at the argument values.
cudaError_t add_kernel_node(cudaGraph_t g, cudaGraphNode_t* node, cudaGraphNode_t dep, void* fn, unsigned grid,
                            unsigned block, void** args) {
    cudaKernelNodeParams kp = {};
    kp.func = fn;
    kp.gridDim = dim3(grid);
    kp.blockDim = dim3(block);
    kp.sharedMemBytes = 0;
    kp.kernelParams = args;
    kp.extra = nullptr;
    return cudaGraphAddKernelNode(node, g, dep ? &dep : nullptr, dep ? 1 : 0, &kp);
}

// The batch-wide PCG graph: graph_iters iterations (even) of the three kernels, built node by node
// (no stream capture, so other host threads that launch work meanwhile cannot disturb it).
int ensure_graph(pms_batch* b) {
    const int gi = std::max(2, b->tune.graph_iters + (b->tune.graph_iters & 1));  // even
    if (b->graph && b->graph_iters_captured == gi) return PMS_OK;
    std::lock_guard<std::mutex> lock(device_mutex());
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaGraph_t g;
    if (cudaGraphCreate(&g, 0) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "graph creation failed");
    const unsigned nch = (unsigned)b->nchunk;
    void* spmv = tpr_of(b->v.nd) == 8 ? (void*)pcg_spmv_dot_kernel<8> : (void*)pcg_spmv_dot_kernel<16>;
    const unsigned qthreads = tpr_of(b->v.nd) == 8 ? quarter_threads<8>() : quarter_threads<16>();
    cudaGraphNode_t prev = nullptr;
    bool ok = true;
    for (int i = 0; i < gi && ok; i++) {
        int par = i & 1;
        const double* val = b->d_csr;
        double rtol = b->cfg.pcg_rtol;
        int32_t max_iter = b->cfg.pcg_max_iterations;
        const int64_t* bptr = b->v.d_bptr;
        const int32_t* bcol = b->v.d_bcol;
        void* a1[] = {&b->S, &par, (void*)&bptr, (void*)&bcol, (void*)&val, &b->d_p, &b->d_q,
                      &b->d_part_c};
        void* a2[] = {&b->S, &par, &b->d_part_c, &b->d_rho, &b->d_p, &b->d_q, &b->d_binv, &b->d_x, &b->d_r,
                      &b->d_z, &b->d_part_a, &b->d_part_b, &b->d_nactive};
        void* a3[] = {&b->S, &par, &b->d_part_a, &b->d_part_b, &b->d_rho, &b->d_r0, &rtol, &max_iter,
                      &b->d_iters, &b->d_z, &b->d_p, &b->d_nactive};
        cudaGraphNode_t n1, n2, n3;
        ok = add_kernel_node(g, &n1, prev, spmv, 4 * nch, qthreads, a1) == cudaSuccess &&
             add_kernel_node(g, &n2, n1, (void*)pcg_update_kernel, nch, CHN, a2) == cudaSuccess &&
             add_kernel_node(g, &n3, n2, (void*)pcg_beta_direction_kernel, nch, CHN, a3) == cudaSuccess;
        prev = n3;
        b->launches += 3;
    }
    if (!ok || cudaGraphInstantiate(&b->graph, g, 0) != cudaSuccess) {
        b->graph = nullptr;
        cudaGraphDestroy(g);
        return bfail(b, PMS_ERR_CUDA, "graph construction failed");
    }
    cudaGraphDestroy(g);
    b->graph_iters_captured = gi;
    return PMS_OK;
}

constexpr int NCLASS = 5;  // team sizes 1, 2, 4, 8, 16

template <int BD, int TPR>
cudaError_t launch_team_t(pms_batch* b, const int32_t* list, int n, int C, int budget, cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(n * C));
    cfg.blockDim = dim3(BD);
    cfg.dynamicSmemBytes = team_smem_bytes(b->v.nd, BD);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)C;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, pcg_team_kernel<BD, TPR>, b->S, list, b->v.d_bptr, b->v.d_bcol,
                              (const double*)b->d_csr, (const double*)b->d_binv, b->d_x, b->d_r, b->d_z, b->d_p,
                              b->d_rho, (const double*)b->d_r0, b->d_iters, b->d_cta_active, b->cfg.pcg_rtol,
                              b->cfg.pcg_max_iterations, budget);
}

int launch_team(pms_batch* b, const int32_t* list, int n, int C, int budget, cudaStream_t st) {
    const bool two = tpr_of(b->v.nd) == 8;
    cudaError_t e;
    switch (b->tune.team_threads) {
        case 256: e = two ? launch_team_t<256, 8>(b, list, n, C, budget, st) : launch_team_t<256, 16>(b, list, n, C, budget, st); break;
        case 1024: e = two ? launch_team_t<1024, 8>(b, list, n, C, budget, st) : launch_team_t<1024, 16>(b, list, n, C, budget, st); break;
        default: e = two ? launch_team_t<512, 8>(b, list, n, C, budget, st) : launch_team_t<512, 16>(b, list, n, C, budget, st); break;
    }
    b->launches++;
    return e == cudaSuccess ? PMS_OK : bfail(b, PMS_ERR_CUDA, cudaGetErrorString(e));
}

template <int BD, int TPR>
bool team_attrs_t() {
    const int sm = (int)team_smem_bytes(TPR == 8 ? 2 : 3, BD);
    return cudaFuncSetAttribute(pcg_team_kernel<BD, TPR>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) ==
               cudaSuccess &&
           cudaFuncSetAttribute(pcg_team_kernel<BD, TPR>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) ==
               cudaSuccess;
}

// Kernel attributes of every team variant, and the largest cluster this device schedules
// (16 where the non-portable size is available, else 8).  Once per process.
int team_setup(int* cmax) {
    static int cached = -1;
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    if (cached < 0) {
        const bool ok = team_attrs_t<256, 8>() && team_attrs_t<256, 16>() && team_attrs_t<512, 8>() &&
                        team_attrs_t<512, 16>() && team_attrs_t<1024, 8>() && team_attrs_t<1024, 16>();
        if (!ok) return PMS_ERR_CUDA;
        int c = 16;
        for (int nd = 2; nd <= 3; nd++) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(16);
            cfg.blockDim = dim3(1024);
            cfg.dynamicSmemBytes = team_smem_bytes(nd, 1024);
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = 16;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int n16 = 0;
            const cudaError_t e = (nd == 2) ? cudaOccupancyMaxActiveClusters(&n16, pcg_team_kernel<1024, 8>, &cfg)
                                            : cudaOccupancyMaxActiveClusters(&n16, pcg_team_kernel<1024, 16>, &cfg);
            if (e != cudaSuccess) cudaGetLastError();
            if (e != cudaSuccess || n16 < 1) c = 8;
        }
        cached = c;
    }
    *cmax = cached;
    return PMS_OK;
}

// Team size of a problem: the smallest power of two whose CTAs hold at most the target number of
// chunks each; 0 (batch-wide engine) when it needs more than the largest cluster.
int team_size_of(const pms_batch* b, int p);

// Which engine runs each problem's PCG (host and device copies): 0 = batch-wide, C = a team of C.
int assign_engines(pms_batch* b) {
    for (int p = 0; p < b->np; p++) b->engine[p] = (b->pndof[p] <= b->tune.team_max_ndof) ? team_size_of(b, p) : 0;
    return cudaMemcpyAsync(b->d_engine, b->engine.data(), b->np, cudaMemcpyHostToDevice, b->v.stream) ==
                   cudaSuccess
               ? PMS_OK
               : bfail(b, PMS_ERR_CUDA, "engine upload failed");
}

// Starts the PCG of the problems selected in d_active: preconditioner, prescribed increments,
// r = R_f - K_fp mdu_p, z, p and the scalars.
void pcg_start(pms_batch* b) {
    cudaStream_t st = b->v.stream;
    block_jacobi_kernel<<<grid_of(b->nnode), 256, 0, st>>>(b->S, b->v.d_bptr, b->v.d_kdiag, b->d_csr, b->d_binv);
    pres_increment_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_u, b->d_c, b->d_mdu);
    launch_spmv(b, b->d_mdu, b->d_kt, b->d_active, false);
    pcg_start_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_rr, b->d_kt, b->d_binv, b->d_r, b->d_x, b->d_z,
                                                           b->d_p, b->d_part_a, b->d_part_b);
    pcg_init_scalars_kernel<<<(unsigned)b->np, CHN, 0, st>>>(b->np, b->d_active, b->d_engine, b->d_pchunk,
                                                                  b->d_part_a, b->d_part_b, b->d_rho, b->d_r0,
                                                                  b->d_pcg_active, b->d_cta_active, b->d_iters);
    b->launches += 4;
}

// PCG iterations of every solving problem: one team launch per team size (each on its own stream)
// and the batch-wide engine (graph launches on the handle's stream) run side by side.  The team
// lists are in b->h_list, grouped by team size (b->cls_off).  The batch-wide loop keeps going while
// a team launch is busy; once they are idle, it stops when an eighth of its problems (at least
// one) have finished or after `budget` iterations.  `exact` runs exactly `budget` iterations on
// every engine (timing).
int pcg_phase(pms_batch* b, int nteam, int nwide, int budget, bool exact) {
    cudaStream_t st = b->v.stream;
    bool launched[NCLASS] = {};
    if (nteam > 0) {
        cudaMemcpyAsync(b->d_list, b->h_list.data(), nteam * 4, cudaMemcpyHostToDevice, st);
        if (cudaEventRecord(b->ev_fork, st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "stream fork failed");
        for (int c = 0; c < NCLASS; c++) {
            const int n = b->cls_off[c + 1] - b->cls_off[c];
            if (n == 0) continue;
            if (cudaStreamWaitEvent(b->st_cls[c], b->ev_fork, 0) != cudaSuccess)
                return bfail(b, PMS_ERR_CUDA, "stream fork failed");
            int rc = launch_team(b, b->d_list + b->cls_off[c], n, 1 << c, budget, b->st_cls[c]);
            if (rc) return rc;
            if (cudaEventRecord(b->ev_cls[c], b->st_cls[c]) != cudaSuccess)
                return bfail(b, PMS_ERR_CUDA, "stream join failed");
            launched[c] = true;
        }
    }
    auto teams_busy = [&]() {
        for (int c = 0; c < NCLASS; c++)
            if (launched[c] && cudaEventQuery(b->ev_cls[c]) == cudaErrorNotReady) return true;
        return false;
    };
    if (nwide > 0) {
        int rc = ensure_graph(b);
        if (rc) return rc;
        int32_t nact = nwide;
        const int32_t stop_at = nwide - std::max(1, nwide / 8);
        for (int64_t done = 0; nact > 0;) {
            if (exact && done >= budget) break;
            if (cudaGraphLaunch(b->graph, st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "graph launch failed");
            done += b->graph_iters_captured;
            if (exact) continue;
            cudaMemcpyAsync(&nact, b->d_nactive, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
            b->host_syncs++;
            if (cudaStreamSynchronize(st) != cudaSuccess)
                return bfail(b, PMS_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
            if (!teams_busy() && (nact <= stop_at || done >= budget)) break;
        }
    }
    for (int c = 0; c < NCLASS; c++)
        if (launched[c] && cudaStreamWaitEvent(st, b->ev_cls[c], 0) != cudaSuccess)
            return bfail(b, PMS_ERR_CUDA, "stream join failed");
    return PMS_OK;
}

// Team lists of the problems selected by `want` (grouped by team size) and the count of
// batch-wide ones.
void build_lists(pms_batch* b, const std::vector<uint8_t>& want, int& nteam, int& nwide) {
    b->h_list.clear();
    nwide = 0;
    for (int c = 0; c < NCLASS; c++) {
        b->cls_off[c] = (int)b->h_list.size();
        for (int p = 0; p < b->np; p++)
            if (want[p] && b->engine[p] == (1 << c)) b->h_list.push_back(p);
    }
    b->cls_off[NCLASS] = (int)b->h_list.size();
    for (int p = 0; p < b->np; p++)
        if (want[p] && b->engine[p] == 0) nwide++;
    nteam = (int)b->h_list.size();
}

int team_size_of(const pms_batch* b, int p) {
    const int64_t nch = b->pnch[p];
    const int cap = team_node_capacity(b->v.nd, b->tune.team_threads) / CHN;
    const int per = b->tune.team_chunks > 0 ? std::min(cap, b->tune.team_chunks) : cap;
    if (nch > TEAM_MAX_CHUNKS) return 0;
    for (int c = 1; c <= b->team_cmax; c *= 2)
        if ((nch + c - 1) / c <= per) return c;
    return 0;
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
    b->tune.team_max_ndof = INT64_MAX;
    b->tune.team_threads = 1024;
    b->tune.team_chunks = 1;
    b->tune.pcg_budget = 128;
    b->tune.graph_iters = 8;
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
    b->pndof.assign(nproblem, 0);
    for (int p = 0; p < nproblem; p++) {
        for (int64_t i = point_ptr[p]; i < point_ptr[p + 1]; i++) node_prob[i] = p;
        for (int64_t c = cell_ptr[p]; c < cell_ptr[p + 1]; c++) cell_prob[c] = p;
        pchunk[p] = (int64_t)chunk_node0.size();
        for (int64_t i = point_ptr[p]; i < point_ptr[p + 1]; i += CHN) {
            chunk_node0.push_back(i);
            chunk_nnode.push_back((int32_t)std::min<int64_t>(CHN, point_ptr[p + 1] - i));
            chunk_prob.push_back(p);
        }
        b->pndof[p] = (point_ptr[p + 1] - point_ptr[p]) * nd;
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
              b->alloc(&b->d_list, nproblem) && b->alloc(&b->d_active, nproblem) &&
              b->alloc(&b->d_pcg_active, 2 * (size_t)nproblem) && b->alloc(&b->d_cta_active, nproblem) &&
              b->alloc(&b->d_pmode, nproblem) && b->alloc(&b->d_first, nproblem) &&
              b->alloc(&b->d_upd, nproblem) && b->alloc(&b->d_engine, nproblem) && b->alloc(&b->d_u, n) &&
              b->alloc(&b->d_ddu, n) && b->alloc(&b->d_ff, n) && b->alloc(&b->d_csr, (size_t)b->v.nnz) &&
              b->alloc(&b->d_rr, n) && b->alloc(&b->d_mdu, n) && b->alloc(&b->d_mdu0, n) &&
              b->alloc(&b->d_kt, n) && b->alloc(&b->d_r, n) && b->alloc(&b->d_z, n) && b->alloc(&b->d_p, n) &&
              b->alloc(&b->d_q, n) && b->alloc(&b->d_x, n) && b->alloc(&b->d_binv, (size_t)b->nnode * nd * nd) &&
              b->alloc(&b->d_lam, npres) && b->alloc(&b->d_c, npres) && b->alloc(&b->d_mdl, npres) &&
              b->alloc(&b->d_mdl0, npres) && b->alloc(&b->d_part_a, b->nchunk) &&
              b->alloc(&b->d_part_b, b->nchunk) && b->alloc(&b->d_part_c, 4 * (size_t)b->nchunk) &&
              b->alloc(&b->d_rho, 2 * (size_t)nproblem) && b->alloc(&b->d_r0, nproblem) &&
              b->alloc(&b->d_norm, nproblem) && b->alloc(&b->d_rel, nproblem) &&
              b->alloc(&b->d_iters, 2 * (size_t)nproblem) &&
              b->alloc(&b->d_nactive, 1) && b->alloc(&b->d_queue, 4 * ((size_t)nproblem + 1)) &&
              b->alloc(&b->d_perr, (size_t)nproblem) && b->alloc(&b->d_phase, nproblem) &&
              b->alloc(&b->d_sel, nproblem) && b->alloc(&b->d_zero_engine, nproblem) &&
              b->alloc(&b->d_st, nproblem) && b->alloc(&b->d_cnt, nproblem) && b->alloc(&b->d_pcgsum, nproblem) &&
              b->alloc(&b->d_it, nproblem) && b->alloc(&b->d_lastnorm, nproblem);
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
    bool sok = cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess &&
               team_setup(&b->team_cmax) == PMS_OK;
    for (int c = 0; c < NCLASS && sok; c++)
        sok = cudaStreamCreateWithFlags(&b->st_cls[c], cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->ev_cls[c], cudaEventDisableTiming) == cudaSuccess;
    if (!sok) {
        delete b;
        return PMS_ERR_CUDA;
    }
    cudaMemset(b->d_u, 0, n * 8);
    cudaMemset(b->d_ddu, 0, n * 8);
    cudaMemset(b->d_lam, 0, std::max<int64_t>(npres, 1) * 8);
    cudaMemset(b->d_p, 0, n * 8);
    cudaMemset(b->d_pcg_active, 0, 2 * (size_t)nproblem);
    cudaMemset(b->d_cta_active, 0, nproblem);
    cudaMemset(b->d_zero_engine, 0, nproblem);
    b->S.nd = nd;
    b->S.np = nproblem;
    b->S.engine = b->d_engine;
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
    b->solving.assign(nproblem, 0);
    b->engine.assign(nproblem, 0);
    b->it.assign(nproblem, 0);
    b->pnch.assign(nproblem, 0);
    for (int p = 0; p < nproblem; p++) b->pnch[p] = pchunk[p + 1] - pchunk[p];
    if (assign_engines(b) || cudaDeviceSynchronize() != cudaSuccess) {
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
    cudaMemsetAsync(b->d_pcg_active, 0, 2 * (size_t)b->np, st);
    cudaMemsetAsync(b->d_cta_active, 0, b->np, st);
    std::fill(b->solving.begin(), b->solving.end(), 0);
    std::fill(b->it.begin(), b->it.end(), 0);
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
    std::vector<uint8_t> elem(np, 0), mode(np, 0), start(np, 0), sel(np, 0), upd(np, 0), first(np, 0);
    std::vector<int32_t> pcg_step(np, 0);
    std::vector<double> hnorm(np, 0.0), hrel(np, 0.0);
    bool any_elem = false;
    for (int p = 0; p < np; p++) {
        result[p] = -1;
        if (cmd[p] == 0 || b->solving[p]) continue;  // solving problems go on with their PCG below
        if (cmd[p] == 1) {
            b->it[p] = 0;
            start[p] = 1;
        }
        elem[p] = 1;
        // mode 1: step start (K assembled); 2: update, F_int and K; 3: constant tangent, K kept
        mode[p] = cmd[p] == 1 ? 1 : (b->cfg.constant_tangent ? 3 : 2);
        any_elem = true;
    }
    if (b->npres > 0) cudaMemcpyAsync(b->d_c, c_values, b->npres * 8, cudaMemcpyHostToDevice, st);
    int rc;
    // ---- stage 1: element pass, residual and its test for the problems that need them
    if (any_elem) {
        cudaMemcpyAsync(b->d_upd, start.data(), np, cudaMemcpyHostToDevice, st);
        zero_masked_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_upd, b->d_ddu);  // new step: dU = 0
        cudaMemcpyAsync(b->d_pmode, mode.data(), np, cudaMemcpyHostToDevice, st);
        // work queue: the cell and node ranges of these problems only
        const size_t W = (size_t)np + 1;
        b->h_queue.assign(4 * W, 0);
        WorkQueue q;
        for (int p = 0; p < np; p++) {
            if (!elem[p]) continue;
            const int k = q.nq++;
            b->h_queue[k + 1] = b->h_queue[k] + (b->cell_ptr[p + 1] - b->cell_ptr[p]);
            b->h_queue[W + k] = b->cell_ptr[p];
            b->h_queue[2 * W + k + 1] = b->h_queue[2 * W + k] + (b->point_ptr[p + 1] - b->point_ptr[p]);
            b->h_queue[3 * W + k] = b->point_ptr[p];
        }
        q.ncell = b->h_queue[q.nq];
        q.nnode = b->h_queue[2 * W + q.nq];
        q.cell_off = b->d_queue;
        q.cell_first = b->d_queue + W;
        q.node_off = b->d_queue + 2 * W;
        q.node_first = b->d_queue + 3 * W;
        cudaMemcpyAsync(b->d_queue, b->h_queue.data(), 4 * W * 8, cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(b->d_perr, 0, (size_t)np * 8, st);
        rc = elements_run_modes(b->el, b->d_cell_prob, b->d_node_prob, b->d_pmode, b->d_ddu, b->d_ff, b->d_csr, &q,
                                b->d_perr);
        if (rc) return rc;
        cudaMemcpyAsync(b->d_active, elem.data(), np, cudaMemcpyHostToDevice, st);
        residual_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_ff, b->d_fext, b->d_u, b->d_lam, b->d_c,
                                                             b->d_rr, b->d_part_a);
        finalize_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_pchunk, b->d_part_a, b->d_norm, 0);
        cudaMemcpyAsync(hnorm.data(), b->d_norm, np * 8, cudaMemcpyDeviceToHost, st);
        std::vector<unsigned long long> perr(np, 0);
        cudaMemcpyAsync(perr.data(), b->d_perr, (size_t)np * 8, cudaMemcpyDeviceToHost, st);
        b->host_syncs++;
        if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "residual failed");
        b->launches += 4;
        // a material or geometry error stops its own problem only; every failing problem of this
        // pass is stopped with the error its own element loop would report first
        rc = elements_status(b->el);
        if (rc != PMS_OK && rc != PMS_ERR_ZERO_SIGMA_D && rc != PMS_ERR_ZERO_NORM_S && rc != PMS_ERR_JACOBIAN)
            return rc;
        for (int p = 0; p < np; p++) {
            if (!elem[p] || perr[p] == 0) continue;
            const int code = decode_error(perr[p], nullptr, nullptr);
            if (code == PMS_ERR_ZERO_SIGMA_D || code == PMS_ERR_ZERO_NORM_S || code == PMS_ERR_JACOBIAN) {
                result[p] = 100 + 1 + code;  // 104: zero sigma_d, 105: zero norm_s, 106: Jacobian
                elem[p] = 0;
            }
        }
        bool any_start = false;
        for (int p = 0; p < np; p++) {
            if (!elem[p]) continue;
            if (iteration) iteration[p] = b->it[p];
            if (norm_rr) norm_rr[p] = hnorm[p];
            if (!std::isfinite(hnorm[p])) {
                result[p] = 101;  // "Found NaN or Inf"
            } else if (hnorm[p] < b->cfg.tol_rr_abs) {
                result[p] = 1;
            } else {
                sel[p] = 1;  // needs the linear solve
                b->solving[p] = 1;
                any_start = true;
            }
        }
        // ---- stage 2: start the linear solve (mdu, mdl) of those problems
        if (any_start) {
            cudaMemcpyAsync(b->d_active, sel.data(), np, cudaMemcpyHostToDevice, st);
            pcg_start(b);
        }
    }
    // ---- stage 3: PCG iterations of every solving problem
    int nteam = 0, nwide = 0;
    build_lists(b, b->solving, nteam, nwide);
    if (nteam + nwide > 0) {
        rc = pcg_phase(b, nteam, nwide, std::max(1, b->tune.pcg_budget), false);
        if (rc) return rc;
        std::vector<uint8_t> wa(np), ca(np);
        cudaMemcpyAsync(wa.data(), b->d_pcg_active, np, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(ca.data(), b->d_cta_active, np, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(pcg_step.data(), b->d_iters, np * 4, cudaMemcpyDeviceToHost, st);
        b->host_syncs++;
        if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "PCG failed");
        // ---- stage 4: problems whose PCG finished complete their Newton iteration
        bool any_fin = false;
        for (int p = 0; p < np; p++) {
            sel[p] = 0;
            if (!b->solving[p]) continue;
            if (wa[p] || ca[p]) {
                result[p] = 2;  // still solving
                continue;
            }
            sel[p] = 1;
            first[p] = (b->it[p] == 0);
            any_fin = true;
        }
        if (any_fin) {
            cudaMemcpyAsync(b->d_active, sel.data(), np, cudaMemcpyHostToDevice, st);
            assemble_mdu_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_x, b->d_mdu);
            if (b->npres > 0)
                multiplier_kernel<<<grid_of(b->npres), 256, 0, st>>>(b->npres, b->d_pres_eq, b->d_pres_prob,
                                                                      b->d_active, b->d_indptr, b->d_indices,
                                                                      b->d_csr, b->d_mdu, b->d_rr, b->d_mdl);
            cudaMemcpyAsync(b->d_first, first.data(), np, cudaMemcpyHostToDevice, st);
            rel_mdu_kernel<<<(unsigned)b->nchunk, CHN, 0, st>>>(b->S, b->d_first, b->d_mdu, b->d_mdu0, b->d_part_a);
            finalize_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_pchunk, b->d_part_a, b->d_rel, 0);
            rel_multipliers_kernel<<<grid_of(np, 128), 128, 0, st>>>(np, b->d_active, b->d_first, b->d_ppres,
                                                                      b->d_mdl, b->d_mdl0, b->d_rel);
            cudaMemcpyAsync(hrel.data(), b->d_rel, np * 8, cudaMemcpyDeviceToHost, st);
            b->host_syncs++;
            if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "solve failed");
            for (int p = 0; p < np; p++) {
                if (!sel[p]) continue;
                b->solving[p] = 0;
                if (iteration) iteration[p] = b->it[p];
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
                update_multipliers_kernel<<<grid_of(b->npres), 256, 0, st>>>(b->npres, b->d_pres_prob, b->d_upd,
                                                                              b->d_mdl, b->d_lam);
            b->launches += 7;
        }
    }
    b->host_syncs++;
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
            pcg_sum[p] += pcg[p];
            if (res[p] == 2) {  // linear solve still under way
                cmd[p] = 2;
                continue;
            }
            count[p] += 1;  // one Newton iteration (residual evaluation, as the reference counts them)
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

}  // extern "C"

namespace {
// Kernel nodes appended one after another to a graph.
struct GraphChain {
    cudaGraph_t g;
    cudaGraphNode_t prev = nullptr;
    bool ok = true;
    int nodes = 0;
    void kernel(const void* fn, unsigned grid, unsigned block, void** args) {
        if (!ok) return;
        cudaGraphNode_t n;
        ok = add_kernel_node(g, &n, prev, (void*)fn, grid, block, args) == cudaSuccess;
        if (ok) {
            prev = n;
            nodes++;
        }
    }
    // a conditional WHILE node on handle h (created on this graph); returns its body graph
    cudaGraph_t while_node(cudaGraphConditionalHandle h) {
        if (!ok) return nullptr;
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t n;
        ok = cudaGraphAddNode(&n, g, prev ? &prev : nullptr, prev ? 1 : 0, &cp) == cudaSuccess;
        if (!ok) return nullptr;
        prev = n;
        return cp.conditional.phGraph_out[0];
    }
};

// The load-step graph (built once per batch; every pointer and constant it uses is fixed).
int build_step_graph(pms_batch* b) {
    if (b->step_graph) return PMS_OK;
    std::lock_guard<std::mutex> lock(device_mutex());
    cudaGraph_t G;
    if (cudaGraphCreate(&G, 0) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "graph creation failed");
    int np = b->np;
    int64_t npres = b->npres;
    SolverArgs S = b->S;
    S.engine = b->d_zero_engine;  // every PCG on the batch-wide engine (the engines give the same bits)
    double tol_rr = b->cfg.tol_rr_abs, tol_mdu = b->cfg.tol_mdu_rel, rtol = b->cfg.pcg_rtol;
    int32_t max_it = b->cfg.n_max_iterations, max_pcg = b->cfg.pcg_max_iterations;
    int zero = 0;
    bool no_mask = false;
    const unsigned nch = (unsigned)b->nchunk;
    const int tpr = tpr_of(b->v.nd);
    const void* spmv_dot = tpr == 8 ? (const void*)pcg_spmv_dot_kernel<8> : (const void*)pcg_spmv_dot_kernel<16>;
    const unsigned qthreads = tpr == 8 ? quarter_threads<8>() : quarter_threads<16>();
    const void* spmv = tpr == 8 ? (const void*)spmv_kernel<8> : (const void*)spmv_kernel<16>;
    const int64_t* bptr = b->v.d_bptr;
    const int32_t* kdiag = b->v.d_kdiag;
    const int32_t* bcol = b->v.d_bcol;
    const double* csr = b->d_csr;
    const double* fext = b->d_fext;
    GraphChain top{G};
    void* a_init[] = {&np, &b->d_sel, &b->d_phase, &b->d_st, &b->d_cnt, &b->d_pcgsum, &b->d_lastnorm};
    top.kernel((const void*)step_init_kernel, 1, 1024, a_init);
    cudaGraphConditionalHandle hN = 0, hP = 0;
    if (top.ok) top.ok = cudaGraphConditionalHandleCreate(&hN, G, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    cudaGraph_t B1 = top.while_node(hN);
    GraphChain body{B1};
    body.ok = top.ok;
    if (body.ok) body.ok = cudaGraphConditionalHandleCreate(&hP, B1, 0, 0) == cudaSuccess;
    // element pass of the problems that start a step or continue it
    int ct = b->cfg.constant_tangent ? 1 : 0;
    void* a_pre[] = {&np, &b->d_phase, &b->d_pmode, &b->d_upd, &b->d_active, &b->d_it, &b->d_perr, &ct};
    body.kernel((const void*)step_pre_elem_kernel, 1, 1024, a_pre);
    void* a_zero[] = {&S, &b->d_upd, &b->d_ddu};
    body.kernel((const void*)zero_masked_kernel, grid_of(b->ndof), 256, a_zero);
    if (body.ok)
        body.ok = elements_graph_pass(b->el, B1, body.prev, &body.prev, b->d_cell_prob, b->d_pmode, b->d_ddu, b->d_ff,
                                      b->d_csr, b->d_perr) == PMS_OK;
    // residual and its tests
    void* a_res[] = {&S, &b->d_ff, (void*)&fext, &b->d_u, &b->d_lam, &b->d_c, &b->d_rr, &b->d_part_a};
    body.kernel((const void*)residual_kernel, nch, CHN, a_res);
    void* a_fin_n[] = {&np, &b->d_pchunk, &b->d_part_a, &b->d_norm, &zero};
    body.kernel((const void*)finalize_kernel, grid_of(np, 128), 128, a_fin_n);
    void* a_post[] = {&np, &hP, &tol_rr, &b->d_perr, &b->d_norm, &b->d_phase, &b->d_active, &b->d_first, &b->d_it,
                      &b->d_st, &b->d_cnt, &b->d_lastnorm};
    body.kernel((const void*)step_post_resid_kernel, 1, 1024, a_post);
    // PCG start (block Jacobi, prescribed increments, r = R_f - K_fp mdu_p, scalars)
    void* a_bj[] = {&S, (void*)&bptr, (void*)&kdiag, (void*)&csr, &b->d_binv};
    body.kernel((const void*)block_jacobi_kernel, grid_of(b->nnode), 256, a_bj);
    void* a_pi[] = {&S, &b->d_u, &b->d_c, &b->d_mdu};
    body.kernel((const void*)pres_increment_kernel, grid_of(b->ndof), 256, a_pi);
    void* a_kt[] = {&S, &b->d_indptr, &b->d_indices, (void*)&csr, &b->d_mdu, &b->d_kt, &b->d_active, &no_mask};
    body.kernel(spmv, grid_of(b->ndof * tpr), 256, a_kt);
    void* a_ps[] = {&S, &b->d_rr, &b->d_kt, &b->d_binv, &b->d_r, &b->d_x, &b->d_z, &b->d_p, &b->d_part_a, &b->d_part_b};
    body.kernel((const void*)pcg_start_kernel, nch, CHN, a_ps);
    void* a_is[] = {&np, &b->d_active, &b->d_zero_engine, &b->d_pchunk, &b->d_part_a, &b->d_part_b, &b->d_rho,
                    &b->d_r0, &b->d_pcg_active, &b->d_cta_active, &b->d_iters};
    body.kernel((const void*)pcg_init_scalars_kernel, (unsigned)np, CHN, a_is);
    // PCG iterations, two per pass (the scalars are double-buffered by iteration parity)
    cudaGraph_t B2 = body.while_node(hP);
    GraphChain pcg{B2};
    pcg.ok = body.ok;
    int par0 = 0, par1 = 1;
    for (int k = 0; k < 2; k++) {
        int* par = k ? &par1 : &par0;
        void* a1[] = {&S, par, (void*)&bptr, (void*)&bcol, (void*)&csr, &b->d_p, &b->d_q, &b->d_part_c};
        pcg.kernel(spmv_dot, 4 * nch, qthreads, a1);
        void* a2[] = {&S, par, &b->d_part_c, &b->d_rho, &b->d_p, &b->d_q, &b->d_binv, &b->d_x, &b->d_r, &b->d_z,
                      &b->d_part_a, &b->d_part_b, &b->d_nactive};
        pcg.kernel((const void*)pcg_update_kernel, nch, CHN, a2);
        void* a3[] = {&S, par, &b->d_part_a, &b->d_part_b, &b->d_rho, &b->d_r0, &rtol, &max_pcg, &b->d_iters, &b->d_z,
                      &b->d_p, &b->d_nactive};
        pcg.kernel((const void*)pcg_beta_direction_kernel, nch, CHN, a3);
    }
    void* a_cp[] = {&hP, &b->d_nactive};
    pcg.kernel((const void*)step_cond_pcg_kernel, 1, 1, a_cp);
    body.ok = body.ok && pcg.ok;
    // completion: mdu, multiplier increments, rel(mdu), and the update
    void* a_am[] = {&S, &b->d_x, &b->d_mdu};
    body.kernel((const void*)assemble_mdu_kernel, grid_of(b->ndof), 256, a_am);
    if (npres > 0) {
        void* a_ml[] = {&npres, &b->d_pres_eq, &b->d_pres_prob, &b->d_active, &b->d_indptr, &b->d_indices,
                        (void*)&csr, &b->d_mdu, &b->d_rr, &b->d_mdl};
        body.kernel((const void*)multiplier_kernel, grid_of(npres), 256, a_ml);
    }
    void* a_rm[] = {&S, &b->d_first, &b->d_mdu, &b->d_mdu0, &b->d_part_a};
    body.kernel((const void*)rel_mdu_kernel, nch, CHN, a_rm);
    void* a_fin_r[] = {&np, &b->d_pchunk, &b->d_part_a, &b->d_rel, &zero};
    body.kernel((const void*)finalize_kernel, grid_of(np, 128), 128, a_fin_r);
    void* a_rml[] = {&np, &b->d_active, &b->d_first, &b->d_ppres, &b->d_mdl, &b->d_mdl0, &b->d_rel};
    body.kernel((const void*)rel_multipliers_kernel, grid_of(np, 128), 128, a_rml);
    void* a_pc[] = {&np, &max_it, &tol_mdu, &b->d_rel, &b->d_active, &b->d_iters, &b->d_phase, &b->d_upd, &b->d_it,
                    &b->d_st, &b->d_pcgsum};
    body.kernel((const void*)step_post_complete_kernel, 1, 1024, a_pc);
    void* a_up[] = {&S, &b->d_upd, &b->d_mdu, &b->d_u, &b->d_ddu};
    body.kernel((const void*)update_kernel, grid_of(b->ndof), 256, a_up);
    if (npres > 0) {
        void* a_uml[] = {&npres, &b->d_pres_prob, &b->d_upd, &b->d_mdl, &b->d_lam};
        body.kernel((const void*)update_multipliers_kernel, grid_of(npres), 256, a_uml);
    }
    void* a_cn[] = {&np, &hN, &b->d_phase};
    body.kernel((const void*)step_cond_newton_kernel, 1, 1024, a_cn);
    const bool ok = top.ok && body.ok;
    if (!ok || cudaGraphInstantiate(&b->step_graph, G, 0) != cudaSuccess) {
        b->step_graph = nullptr;
        cudaGraphDestroy(G);
        return bfail(b, PMS_ERR_CUDA, "load-step graph construction failed");
    }
    cudaGraphDestroy(G);
    b->launches += top.nodes + body.nodes + pcg.nodes + 1;
    return PMS_OK;
}
}  // namespace

extern "C" {

int pms_batch_solve_step_graph(pms_batch* b, const double* c_values, const uint8_t* active, int32_t* iterations,
                               double* norm_rr, int32_t* status, int32_t* pcg_iterations) {
    if (!b || !active) return PMS_ERR_INVALID;
    if (b->npres > 0 && !c_values) return PMS_ERR_INVALID;
    const int np = b->np;
    for (int p = 0; p < np; p++)
        if (b->solving[p]) return bfail(b, PMS_ERR_INVALID, "a tick-driven linear solve is under way");
    int rc = build_step_graph(b);
    if (rc) return rc;
    cudaStream_t st = b->v.stream;
    if (b->npres > 0) cudaMemcpyAsync(b->d_c, c_values, b->npres * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->d_sel, active, np, cudaMemcpyHostToDevice, st);
    if (cudaGraphLaunch(b->step_graph, st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, "load-step graph launch failed");
    std::vector<int32_t> cnt(np), stv(np), pcg(np), itv(np);
    std::vector<double> norm(np);
    cudaMemcpyAsync(cnt.data(), b->d_cnt, np * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(stv.data(), b->d_st, np * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(pcg.data(), b->d_pcgsum, np * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(itv.data(), b->d_it, np * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(norm.data(), b->d_lastnorm, np * 8, cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return bfail(b, PMS_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    rc = elements_status(b->el);  // element errors are per problem (in stv); anything else is fatal
    if (rc != PMS_OK && rc != PMS_ERR_ZERO_SIGMA_D && rc != PMS_ERR_ZERO_NORM_S && rc != PMS_ERR_JACOBIAN) return rc;
    for (int p = 0; p < np; p++) {
        if (active[p]) b->it[p] = itv[p];
        b->pcg_total += pcg[p];
        if (iterations) iterations[p] = cnt[p];
        if (norm_rr) norm_rr[p] = norm[p];
        if (status) status[p] = stv[p] >= 100 ? stv[p] - 100 : 0;
        if (pcg_iterations) pcg_iterations[p] = pcg[p];
    }
    b->host_syncs += 1;
    return PMS_OK;
}

int64_t pms_batch_host_syncs(const pms_batch* b) { return b ? b->host_syncs : 0; }

int pms_batch_set_tuning(pms_batch* b, const pms_batch_tuning* t) {
    if (!b || !t) return PMS_ERR_INVALID;
    if (t->team_threads != 256 && t->team_threads != 512 && t->team_threads != 1024) return PMS_ERR_INVALID;
    if (t->pcg_budget < 1 || t->graph_iters < 1 || t->graph_iters > 64 || t->team_max_ndof < 0 ||
        t->team_chunks < 0)
        return PMS_ERR_INVALID;
    for (int p = 0; p < b->np; p++)
        if (b->solving[p]) return bfail(b, PMS_ERR_INVALID, "tuning cannot change while a linear solve is under way");
    b->tune = *t;
    if (cudaStreamSynchronize(b->v.stream) != cudaSuccess) return PMS_ERR_CUDA;
    return assign_engines(b);
}

int pms_batch_get_tuning(const pms_batch* b, pms_batch_tuning* t) {
    if (!b || !t) return PMS_ERR_INVALID;
    *t = b->tune;
    return PMS_OK;
}

namespace {

// Sets up every problem's PCG on its initial tangent with a unit right-hand side (after
// pms_batch_reset): step-start element pass, block-Jacobi, r = 1 on the free rows.
int timing_setup(pms_batch* b) {
    for (int p = 0; p < b->np; p++)
        if (b->solving[p]) return bfail(b, PMS_ERR_INVALID, "timing needs a batch with no solve under way");
    cudaStream_t st = b->v.stream;
    const int np = b->np;
    int rc = pms_batch_reset(b);
    if (rc) return rc;
    std::vector<uint8_t> all(np, 1);
    cudaMemcpyAsync(b->d_pmode, all.data(), np, cudaMemcpyHostToDevice, st);
    rc = elements_run_modes(b->el, b->d_cell_prob, b->d_node_prob, b->d_pmode, b->d_ddu, b->d_ff, b->d_csr);
    if (rc) return rc;
    rc = elements_status(b->el);
    if (rc) return rc;
    cudaMemcpyAsync(b->d_active, all.data(), np, cudaMemcpyHostToDevice, st);
    fill_masked_kernel<<<grid_of(b->ndof), 256, 0, st>>>(b->S, b->d_active, b->d_rr, 1.0);
    std::vector<double> zc(std::max<int64_t>(b->npres, 1), 0.0);
    cudaMemcpyAsync(b->d_c, zc.data(), std::max<int64_t>(b->npres, 1) * 8, cudaMemcpyHostToDevice, st);
    return cudaStreamSynchronize(st) == cudaSuccess ? PMS_OK : bfail(b, PMS_ERR_CUDA, "timing setup failed");
}

// Device time (ms) of `iters` PCG iterations of every problem with the given launch shapes (second
// of two runs, the first warms up), after timing_setup.
int time_candidate(pms_batch* b, const pms_batch_tuning& cand, int iters, float* ms_out) {
    cudaStream_t st = b->v.stream;
    const int np = b->np;
    b->tune = cand;
    int rc = assign_engines(b);
    if (rc) return rc;
    std::vector<uint8_t> all(np, 1);
    int nteam = 0, nwide = 0;
    build_lists(b, all, nteam, nwide);
    cudaMemcpyAsync(b->d_active, all.data(), np, cudaMemcpyHostToDevice, st);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float ms = 0.0f;
    for (int rep = 0; rep < 2 && !rc; rep++) {
        pcg_start(b);
        cudaEventRecord(e0, st);
        rc = pcg_phase(b, nteam, nwide, iters, true);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) rc = bfail(b, PMS_ERR_CUDA, "timing run failed");
        cudaEventElapsedTime(&ms, e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_out = ms;
    return rc;
}

}  // namespace

int pms_batch_time_pcg(pms_batch* b, const pms_batch_tuning* t, int32_t iterations, double* ms) {
    if (!b || !t || !ms || iterations < 1) return PMS_ERR_INVALID;
    const pms_batch_tuning keep = b->tune;
    int rc = pms_batch_set_tuning(b, t);
    if (rc) return rc;
    rc = timing_setup(b);
    float m = 0.0f;
    if (!rc) rc = time_candidate(b, *t, iterations, &m);
    *ms = m;
    b->tune = keep;
    int rc2 = assign_engines(b);
    int rc3 = pms_batch_reset(b);
    return rc ? rc : (rc2 ? rc2 : rc3);
}

int pms_batch_autotune(pms_batch* b, pms_batch_tuning* out) {
    if (!b) return PMS_ERR_INVALID;
    int rc = timing_setup(b);
    if (rc) return rc;
    const int np = b->np;
    // candidates: the batch-wide engine alone, then teams for every problem that fits (or only for
    // the problems up to a size) with several CTA sizes and chunks per CTA
    int64_t maxdof = 0;
    for (int p = 0; p < np; p++) maxdof = std::max(maxdof, b->pndof[p]);
    const pms_batch_tuning keep = b->tune;
    std::vector<pms_batch_tuning> cands;
    {
        pms_batch_tuning c = keep;
        c.team_max_ndof = 0;
        cands.push_back(c);
    }
    for (int64_t t : {(int64_t)2048, (int64_t)8192, INT64_MAX}) {
        if (t != INT64_MAX && t >= maxdof) continue;
        for (int threads : {512, 1024})
            for (int chunks : {0, 1, 4}) {
                pms_batch_tuning c = keep;
                c.team_max_ndof = t;
                c.team_threads = threads;
                c.team_chunks = chunks;
                cands.push_back(c);
            }
    }
    pms_batch_tuning best = keep;
    float best_ms = 1e30f;
    for (const auto& cand : cands) {
        float ms = 0.0f;
        rc = time_candidate(b, cand, 32, &ms);
        if (rc) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = cand;
        }
    }
    b->tune = rc ? keep : best;
    int rc2 = assign_engines(b);
    int rc3 = pms_batch_reset(b);
    if (!rc && out) *out = b->tune;
    return rc ? rc : (rc2 ? rc2 : rc3);
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
