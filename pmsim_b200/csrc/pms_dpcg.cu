// Distributed block-Jacobi PCG: one rank's part of a conjugate-gradient solve over the owned rows of
// a sharded stiffness matrix (no counterpart in the reference, which solves one problem in one
// process with a direct solver, src/fem/solver_implicit.rs:187-272).
//
// The rank holds the owned rows of its local K (columns in local DOF numbering: owned DOFs first,
// then ghosts).  The prescribed DOFs are eliminated: their rows and columns are replaced by the
// identity and their right-hand side by 0.  The operator is kept as a CSR over the owned rows,
// split into interior rows (every column owned) and boundary rows (some ghost column), so that the
// ghost exchange of the search direction can run while the interior rows are multiplied.  The
// preconditioner is the inverse of each owned node's ND x ND diagonal block (the batched solver's
// block-Jacobi, spd_block_inverse).
//
// Every dot product is a fixed-shape reduction (a fixed grid; each block sums its nodes by the warp
// tree; the last block to finish adds the block partials in index order), so a rank's partial sums
// are the same bits on every run.  The host adds them across ranks (an all-reduce on the scalar
// slots) between the kernels; the kernels read the reduced values from device memory, so no host
// synchronisation is needed inside an iteration.  Convergence (r.z <= rtol^2 r0.z0) is decided on
// the device from the reduced value, identically on every rank, and freezes the iterates.

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pms.h"
#include "pms_device.cuh"

using namespace pms;

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int DT = 256;        // threads per block of the vector kernels
constexpr int DOT_BLOCKS = 296;  // upper bound of the reduction grid (2 blocks per SM)
constexpr int TPR = 8;           // lanes per row of the SpMV

enum Slot { RZN = 0, PQ = 1, RZ = 2, RZ0 = 3, DONE = 4, ITERS = 5 };

}  // namespace

struct pms_dpcg {
    int nd = 0;
    int64_t n = 0, nl = 0, nnode = 0, nnz = 0;
    int64_t n_in = 0, n_bd = 0, nsend = 0, nrecv = 0;
    int nblk = 1;
    int64_t* d_ptr = nullptr;    // eliminated CSR over the owned rows
    int32_t* d_col = nullptr;
    double* d_val = nullptr;
    int64_t* d_src = nullptr;    // source position of each value in the local CSR values, -1: unit diagonal
    int32_t* d_rows_in = nullptr, * d_rows_bd = nullptr;
    uint8_t* d_fixed = nullptr;  // owned DOFs
    int64_t* d_dpos = nullptr;   // per owned node: [nd][nd] positions of its diagonal block in d_val (-1: none)
    double* d_binv = nullptr;
    int64_t* d_send = nullptr, * d_recv = nullptr;
    double* d_part = nullptr;
    unsigned* d_ticket = nullptr;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr, *sb = nullptr, *rb = nullptr,
           *scal = nullptr;
    cudaStream_t st = nullptr;
    std::string err;
    std::vector<void*> owned;

    template <typename T>
    bool upload(T** d, const T* h, size_t n) {
        if (n == 0) return true;
        if (cudaMalloc(d, n * sizeof(T)) != cudaSuccess) return false;
        owned.push_back(*d);
        return cudaMemcpy(*d, h, n * sizeof(T), cudaMemcpyHostToDevice) == cudaSuccess;
    }
    template <typename T>
    bool alloc(T** d, size_t n) {
        if (cudaMalloc(d, (n ? n : 1) * sizeof(T)) != cudaSuccess) return false;
        owned.push_back(*d);
        return true;
    }
    ~pms_dpcg() {
        for (void* v : owned) cudaFree(v);
    }
    bool bound() const { return x && r && z && p && q && scal && (nsend == 0 || sb) && (nrecv == 0 || rb); }
};

namespace {

std::string& dpcg_create_error() {
    static thread_local std::string msg;
    return msg;
}

// Sum of v over the block by the warp tree, then over the warps in order; thread 0 gets it.
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    return s;
}

// Block partial into part[blockIdx.x]; the last block to arrive adds the partials in index order
// into *out and resets the ticket for the next reduction.
__device__ __forceinline__ void reduce_to(double v, double* sh, double* part, unsigned* ticket, double* out) {
    const double s = block_sum(v, sh);
    __shared__ bool last;
    if (threadIdx.x == 0) {
        part[blockIdx.x] = s;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        double t = 0.0;
        for (unsigned b = 0; b < gridDim.x; b++) t += __ldcg(part + b);
        *out = t;
        *ticket = 0;
    }
}

__device__ __forceinline__ bool is_done(const double* scal) { return scal[DONE] != 0.0; }

__global__ void set_values_kernel(int64_t nnz, const int64_t* src, const double* vals_local, double* val) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nnz) val[k] = src[k] >= 0 ? vals_local[src[k]] : 1.0;
}

__global__ void binv_kernel(int64_t nnode, int nd, const int64_t* dpos, const uint8_t* fixed, const double* val,
                            double* binv) {
    const int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nnode) return;
    double a[3][6];
    int fr[3], nf = 0;
    for (int i = 0; i < nd; i++)
        if (!fixed[node * nd + i]) fr[nf++] = i;
    const int64_t* dp = dpos + node * nd * nd;
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++) {
            const int64_t k = dp[fr[i] * nd + fr[j]];
            a[i][j] = k >= 0 ? val[k] : 0.0;
            a[i][nf + j] = (i == j) ? 1.0 : 0.0;
        }
    const bool ok = spd_block_inverse(a, nf);
    double* out = binv + node * nd * nd;
    for (int i = 0; i < nd * nd; i++) out[i] = 0.0;
    for (int i = 0; i < nf; i++)
        for (int j = 0; j < nf; j++)
            out[fr[i] * nd + fr[j]] = ok ? a[i][nf + j] : (i == j ? 1.0 / fmax(fabs(a[i][i]), 1e-300) : 0.0);
}

// z = B^-1 r on one node; returns its r.z
template <int ND>
__device__ __forceinline__ double precondition(const double* B, const double (&rv)[ND], double (&zv)[ND]) {
    double rz = 0.0;
#pragma unroll
    for (int d = 0; d < ND; d++) {
        double s = 0.0;
#pragma unroll
        for (int e = 0; e < ND; e++) s = fma(B[d * ND + e], rv[e], s);
        zv[d] = s;
        rz = fma(rv[d], s, rz);
    }
    return rz;
}

// x = 0, r = b (0 on prescribed rows), z = M r, p = z; partial r.z into scal[RZN]
template <int ND>
__global__ void start_kernel(int64_t nnode, const uint8_t* fixed, const double* b, const double* binv, double* x,
                             double* r, double* z, double* p, double* part, unsigned* ticket, double* scal) {
    __shared__ double sh[32];
    double acc = 0.0;
    for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < nnode;
         node += (int64_t)gridDim.x * blockDim.x) {
        double rv[ND], zv[ND];
#pragma unroll
        for (int d = 0; d < ND; d++) {
            const int64_t i = node * ND + d;
            rv[d] = fixed[i] ? 0.0 : b[i];
            r[i] = rv[d];
            x[i] = 0.0;
        }
        acc += precondition<ND>(binv + node * ND * ND, rv, zv);
#pragma unroll
        for (int d = 0; d < ND; d++) {
            z[node * ND + d] = zv[d];
            p[node * ND + d] = zv[d];
        }
    }
    reduce_to(acc, sh, part, ticket, scal + RZN);
}

// after the all-reduce of r.z: rz = rz0 = r.z, iterations 0, done when r.z is not positive
__global__ void init_kernel(double* scal) {
    scal[RZ] = scal[RZN];
    scal[RZ0] = scal[RZN];
    scal[ITERS] = 0.0;
    scal[DONE] = scal[RZN] > 0.0 ? 0.0 : 1.0;
}

__global__ void gather_kernel(int64_t n, const int64_t* idx, const double* src, double* dst, const double* scal) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !is_done(scal)) dst[k] = src[idx[k]];
}

__global__ void scatter_kernel(int64_t n, const int64_t* idx, const double* src, double* dst, const double* scal) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n && !is_done(scal)) dst[idx[k]] = src[k];
}

// q = A p on a list of rows, TPR lanes per row: each lane sums its entries in order, then the
// lanes' sums by a shuffle tree (fixed order)
__global__ void spmv_kernel(int64_t nrows, const int32_t* rows, const int64_t* ptr, const int32_t* col,
                            const double* val, const double* p, double* q, const double* scal) {
    const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t k = gid / TPR;
    const int sub = (int)(gid % TPR);
    const bool on = k < nrows && !is_done(scal);
    double s = 0.0;
    int64_t row = 0;
    if (on) {
        row = rows[k];
        for (int64_t e = ptr[row] + sub; e < ptr[row + 1]; e += TPR) s = fma(val[e], p[col[e]], s);
    }
#pragma unroll
    for (int o = TPR / 2; o > 0; o >>= 1) s += __shfl_down_sync(FULL, s, o, TPR);
    if (on && sub == 0) q[row] = s;
}

// partial p.q over the owned DOFs into scal[PQ]
__global__ void dot_pq_kernel(int64_t nnode, int nd, const double* p, const double* q, double* part,
                              unsigned* ticket, double* scal) {
    __shared__ double sh[32];
    double acc = 0.0;
    if (!is_done(scal))
        for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < nnode;
             node += (int64_t)gridDim.x * blockDim.x) {
            double s = 0.0;
            for (int d = 0; d < nd; d++) s = fma(p[node * nd + d], q[node * nd + d], s);
            acc += s;
        }
    reduce_to(acc, sh, part, ticket, scal + PQ);
}

// alpha = rz / p.q (reduced); x += alpha p, r -= alpha q, z = M r; partial r.z into scal[RZN]
template <int ND>
__global__ void update_kernel(int64_t nnode, const double* binv, const double* p, const double* q, double* x,
                              double* r, double* z, double* part, unsigned* ticket, double* scal) {
    __shared__ double sh[32];
    double acc = 0.0;
    const bool done = is_done(scal);
    if (!done) {
        const double alpha = scal[RZ] / scal[PQ];
        for (int64_t node = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; node < nnode;
             node += (int64_t)gridDim.x * blockDim.x) {
            double rv[ND], zv[ND];
#pragma unroll
            for (int d = 0; d < ND; d++) {
                const int64_t i = node * ND + d;
                x[i] = fma(alpha, p[i], x[i]);
                rv[d] = fma(-alpha, q[i], r[i]);
                r[i] = rv[d];
            }
            acc += precondition<ND>(binv + node * ND * ND, rv, zv);
#pragma unroll
            for (int d = 0; d < ND; d++) z[node * ND + d] = zv[d];
        }
    }
    reduce_to(acc, sh, part, ticket, scal + RZN);
}

// p = z + (r.z_new / r.z) p on the owned DOFs
__global__ void direction_kernel(int64_t n, const double* z, double* p, const double* scal) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || is_done(scal)) return;
    const double beta = scal[RZN] / scal[RZ];
    p[i] = fma(beta, p[i], z[i]);
}

// rz = r.z_new, one more iteration; done when r.z_new <= rtol^2 r0.z0
__global__ void scalars_kernel(double* scal, double rtol2) {
    if (scal[DONE] != 0.0) return;
    scal[RZ] = scal[RZN];
    scal[ITERS] += 1.0;
    if (scal[RZN] <= rtol2 * scal[RZ0]) scal[DONE] = 1.0;
}

inline unsigned blocks_for(int64_t n, int t = DT) { return (unsigned)((n + t - 1) / t); }

int launched(pms_dpcg* h) {
    const cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) return PMS_OK;
    h->err = cudaGetErrorString(e);
    return PMS_ERR_CUDA;
}

}  // namespace

extern "C" {

int pms_dpcg_create(int32_t ndim, int64_t n_owned, int64_t n_local, const int64_t* indptr, const int32_t* indices,
                    const uint8_t* fixed_local, int64_t nsend, const int64_t* send_idx, int64_t nrecv,
                    const int64_t* recv_idx, pms_dpcg** out) {
    auto refuse = [](const char* m) {
        dpcg_create_error() = m;
        return PMS_ERR_INVALID;
    };
    if (!out) return refuse("out is NULL");
    *out = nullptr;
    if ((ndim != 2 && ndim != 3) || n_owned < 0 || n_local < n_owned || n_owned % ndim || n_local % ndim)
        return refuse("ndim must be 2 or 3, n_owned <= n_local, both multiples of ndim");
    if (!indptr || (n_owned > 0 && (!indices || !fixed_local)) || nsend < 0 || nrecv < 0 ||
        (nsend && !send_idx) || (nrecv && !recv_idx))
        return refuse("missing array");
    const int nd = ndim;
    const int64_t n = n_owned;
    std::vector<int64_t> ptr(n + 1, 0), src, dpos((size_t)n * nd, -1);
    std::vector<int32_t> col, rin, rbd;
    for (int64_t row = 0; row < n; row++) {
        if (indptr[row + 1] < indptr[row]) return refuse("indptr must not decrease");
        bool ghost = false;
        const int64_t node = row / nd;
        auto keep = [&](int32_t c, int64_t s) {
            if (c / nd == node) dpos[(size_t)node * nd * nd + (row % nd) * nd + c % nd] = (int64_t)col.size();
            col.push_back(c);
            src.push_back(s);
            ghost = ghost || c >= n;
        };
        if (fixed_local[row]) {
            keep((int32_t)row, -1);
        } else {
            for (int64_t k = indptr[row]; k < indptr[row + 1]; k++) {
                const int32_t c = indices[k];
                if (c < 0 || c >= n_local) return refuse("column index out of range");
                if (!fixed_local[c]) keep(c, k);
            }
        }
        ptr[row + 1] = (int64_t)col.size();
        (ghost ? rbd : rin).push_back((int32_t)row);
    }
    for (int64_t k = 0; k < nsend; k++)
        if (send_idx[k] < 0 || send_idx[k] >= n) return refuse("send index must name an owned DOF");
    for (int64_t k = 0; k < nrecv; k++)
        if (recv_idx[k] < n || recv_idx[k] >= n_local) return refuse("receive index must name a ghost DOF");
    auto* h = new pms_dpcg;
    h->nd = nd;
    h->n = n;
    h->nl = n_local;
    h->nnode = n / nd;
    h->nnz = (int64_t)col.size();
    h->n_in = (int64_t)rin.size();
    h->n_bd = (int64_t)rbd.size();
    h->nsend = nsend;
    h->nrecv = nrecv;
    h->nblk = (int)std::max<int64_t>(1, std::min<int64_t>(DOT_BLOCKS, (h->nnode + DT - 1) / DT));
    std::vector<uint8_t> fixed_own(fixed_local, fixed_local + n);
    const bool ok = h->upload(&h->d_ptr, ptr.data(), ptr.size()) && h->upload(&h->d_col, col.data(), col.size()) &&
                    h->upload(&h->d_src, src.data(), src.size()) && h->alloc(&h->d_val, col.size()) &&
                    h->upload(&h->d_rows_in, rin.data(), rin.size()) &&
                    h->upload(&h->d_rows_bd, rbd.data(), rbd.size()) &&
                    h->upload(&h->d_fixed, fixed_own.data(), fixed_own.size()) &&
                    h->upload(&h->d_dpos, dpos.data(), dpos.size()) && h->alloc(&h->d_binv, (size_t)n * nd) &&
                    h->upload(&h->d_send, send_idx, (size_t)nsend) && h->upload(&h->d_recv, recv_idx, (size_t)nrecv) &&
                    h->alloc(&h->d_part, (size_t)h->nblk) && h->alloc(&h->d_ticket, 1) &&
                    cudaMemset(h->d_ticket, 0, sizeof(unsigned)) == cudaSuccess;
    if (!ok) {
        delete h;
        cudaGetLastError();
        dpcg_create_error() = "out of device memory";
        return PMS_ERR_NOMEM;
    }
    dpcg_create_error().clear();
    *out = h;
    return PMS_OK;
}

void pms_dpcg_destroy(pms_dpcg* h) { delete h; }

const char* pms_dpcg_last_error(const pms_dpcg* h) { return h ? h->err.c_str() : dpcg_create_error().c_str(); }

int pms_dpcg_set_stream(pms_dpcg* h, void* stream) {
    if (!h) return PMS_ERR_INVALID;
    h->st = (cudaStream_t)stream;
    return PMS_OK;
}

int pms_dpcg_bind(pms_dpcg* h, double* x, double* r, double* z, double* p, double* q, double* sendbuf, double* recvbuf,
                  double* scal) {
    if (!h) return PMS_ERR_INVALID;
    h->x = x;
    h->r = r;
    h->z = z;
    h->p = p;
    h->q = q;
    h->sb = sendbuf;
    h->rb = recvbuf;
    h->scal = scal;
    if (!h->bound()) {
        h->err = "every vector must be given (send/receive buffers may be NULL when empty)";
        return PMS_ERR_INVALID;
    }
    return PMS_OK;
}

int pms_dpcg_set_values(pms_dpcg* h, const double* values) {
    if (!h || (h->nnz && !values)) return PMS_ERR_INVALID;
    if (h->nnz) set_values_kernel<<<blocks_for(h->nnz), DT, 0, h->st>>>(h->nnz, h->d_src, values, h->d_val);
    if (h->nnode)
        binv_kernel<<<blocks_for(h->nnode, 128), 128, 0, h->st>>>(h->nnode, h->nd, h->d_dpos, h->d_fixed, h->d_val,
                                                                  h->d_binv);
    return launched(h);
}

int pms_dpcg_start(pms_dpcg* h, const double* b) {
    if (!h || !h->bound() || (h->n && !b)) return PMS_ERR_INVALID;
    auto k = h->nd == 2 ? start_kernel<2> : start_kernel<3>;
    k<<<h->nblk, DT, 0, h->st>>>(h->nnode, h->d_fixed, b, h->d_binv, h->x, h->r, h->z, h->p, h->d_part, h->d_ticket,
                                 h->scal);
    return launched(h);
}

int pms_dpcg_init(pms_dpcg* h) {
    if (!h || !h->bound()) return PMS_ERR_INVALID;
    init_kernel<<<1, 1, 0, h->st>>>(h->scal);
    return launched(h);
}

int pms_dpcg_pack(pms_dpcg* h) {
    if (!h || !h->bound()) return PMS_ERR_INVALID;
    if (h->nsend) gather_kernel<<<blocks_for(h->nsend), DT, 0, h->st>>>(h->nsend, h->d_send, h->p, h->sb, h->scal);
    return launched(h);
}

int pms_dpcg_unpack(pms_dpcg* h) {
    if (!h || !h->bound()) return PMS_ERR_INVALID;
    if (h->nrecv) scatter_kernel<<<blocks_for(h->nrecv), DT, 0, h->st>>>(h->nrecv, h->d_recv, h->rb, h->p, h->scal);
    return launched(h);
}

int pms_dpcg_spmv(pms_dpcg* h, int32_t boundary) {
    if (!h || !h->bound() || (boundary != 0 && boundary != 1)) return PMS_ERR_INVALID;
    const int64_t nr = boundary ? h->n_bd : h->n_in;
    const int32_t* rows = boundary ? h->d_rows_bd : h->d_rows_in;
    if (nr) spmv_kernel<<<blocks_for(nr * TPR), DT, 0, h->st>>>(nr, rows, h->d_ptr, h->d_col, h->d_val, h->p, h->q,
                                                                h->scal);
    return launched(h);
}

int pms_dpcg_dot_pq(pms_dpcg* h) {
    if (!h || !h->bound()) return PMS_ERR_INVALID;
    dot_pq_kernel<<<h->nblk, DT, 0, h->st>>>(h->nnode, h->nd, h->p, h->q, h->d_part, h->d_ticket, h->scal);
    return launched(h);
}

int pms_dpcg_update(pms_dpcg* h) {
    if (!h || !h->bound()) return PMS_ERR_INVALID;
    auto k = h->nd == 2 ? update_kernel<2> : update_kernel<3>;
    k<<<h->nblk, DT, 0, h->st>>>(h->nnode, h->d_binv, h->p, h->q, h->x, h->r, h->z, h->d_part, h->d_ticket, h->scal);
    return launched(h);
}

int pms_dpcg_direction(pms_dpcg* h, double rtol) {
    if (!h || !h->bound()) return PMS_ERR_INVALID;
    if (h->n) direction_kernel<<<blocks_for(h->n), DT, 0, h->st>>>(h->n, h->z, h->p, h->scal);
    scalars_kernel<<<1, 1, 0, h->st>>>(h->scal, rtol * rtol);
    return launched(h);
}

int pms_dpcg_info(const pms_dpcg* h, int64_t* counts) {
    if (!h || !counts) return PMS_ERR_INVALID;
    counts[0] = h->nnz;
    counts[1] = h->n_in;
    counts[2] = h->n_bd;
    counts[3] = h->nblk;
    return PMS_OK;
}

}  // extern "C"
