// pms_elements.cu -- fused per-element kernels (strain -> return map -> B^T sigma -> B^T D B)
// and the deterministic CSR / residual gathers, behind the pms_elements_* C ABI.
//
// Reference calls replaced (pmsim 0.3.0):
//   ElementSolid::update_secondary_values  src/fem/element_solid.rs:190-224 (+ calculate_strain,
//                                          src/base/calculate_strain.rs:18-60)
//   ElementSolid::calc_f_int               src/fem/element_solid.rs:124-138 (gemlab integ::vec_04_tb)
//   ElementSolid::calc_jacobian            src/fem/element_solid.rs:168-185 (gemlab integ::mat_10_bdb)
//   Elements::{assemble_f_int, assemble_kke, update_secondary_values, backup, restore, reset}
//                                          src/fem/elements.rs:132-205
//   assemble_vector / assemble_matrix      src/base/assembly.rs:38-139
//
// Work decomposition: one warp per cell.  Lane m < nnode owns node m (coordinates, dU, its
// share of f_int); lane p < ngauss owns the state of integration point p (loaded coalesced at
// the start, broadcast by shuffle when p is processed).  Per IP the warp reduces J and the
// strain increment by shuffles, every lane runs the (identical) return map, and each lane
// accumulates its share of the upper-triangular node-pair blocks of K_e in registers.
//
// Tangent algebra.  The von Mises / Hooke tangent is D = a Psd + b s(x)s + K I(x)I.  With the
// node gradients g_m, h_m = S g_m (S the deviatoric stress tensor) and the Mandel B matrix,
//   B_a^T B_b = 1/2 ((g_a.g_b) 1 + g_b (x) g_a),  B_a^T I = g_a,  B_a^T s = h_a,
// so the 3x3 (2x2) block of node pair (a, b) is
//   K_ab += w|J| [ a/2 (g_a.g_b) 1 + a/2 g_b(x)g_a + (K - a/3) g_a(x)g_b + b h_a(x)h_b ].
// This is B^T D B exactly (same bilinear form), evaluated with 3 FMA per block entry instead of
// forming D and D.B; results agree with the dense product to rounding.
// FLOPs per IP and pair (3D): 3 (dot) + 9*3 (entries) + 3 (diagonal) = 33 FMA; per node: J^-T
// dN (9), h = S g (9), three scaled copies (9).
//
// 2D cells (at most 9 nodes) run in element2d_kernel instead: the same arithmetic with several
// cells per warp (three 10-lane Qua8 cells), so that most lanes hold work.
//
// Assembly: each cell's dense element matrix goes to a scratch buffer ke[cell][NE][NE] (the
// reference's GenericElement::kke, src/fem/elements.rs:13-14); in kk_gather_kernel a group of
// nnode lanes owns one block row A of K (32/nnode rows per warp), adds the node-row slabs (a, all
// b) of the cells incident to A in ascending cell order in shared memory and writes the CSR row
// once, coalesced.  No atomics: bit-identical on every run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/pms.h"
#include "pms_device.cuh"
#include "pms_internal.h"
#include "pms_pattern.h"
#include "pms_shapes.h"

using namespace pms;

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int WPB = 4;  // warps (cells) per block

// Modes of the element kernel
// UPD_MODE: the mode comes at run time from the cell's problem (batched solver):
//   0 = inactive (cell skipped), 1 = step start: assemble from the current state with lambda = 0
//   and copy it to the backup, 2 = update from the backup with ddu, then assemble.
enum { UPD_NONE = 0, UPD_CURRENT = 1, UPD_BACKUP = 2, UPD_MODE = 3 };

struct ElemArgs {
    int64_t ncell;     // cells in this launch
    int64_t cell0;     // first cell of this launch
    int axisym = 0;    // 2D axisymmetric idealization (x = radius)
    int64_t nip;       // total IPs of the mesh (SoA stride)
    int ngauss;
    double thickness;
    const double* coords;   // npoint*nd
    const int32_t* conn;    // ncell_total*nn
    const int32_t* cmat;    // per-cell material (nullable)
    const MatConst* mats;
    const double* ddu;      // ndof
    const double* tab;      // dN[ngauss][nn][nd], then w[ngauss], then N[ngauss][nn] (axisymmetric)
    // IP state, SoA with stride nip: sig[c*nip + ip]
    const double* sig_src; const double* z_src; const double* lam_src; const uint8_t* el_src;
    double* sig; double* z; double* lam; uint8_t* el;
    double* fe;   // [cell][nn][nd]
    double* ke;   // [cell][NE][NE] dense element matrices
    unsigned long long* errkey;  // error key of the failing IP the reference would report (0: none)
    unsigned long long* prob_err = nullptr;  // UPD_MODE (nullable): the same key per problem
    const int32_t* cell_prob = nullptr;  // UPD_MODE: problem of each cell
    const uint8_t* pmode = nullptr;      // UPD_MODE: mode of each problem
    // work queue (nq > 0): the launch covers ncell queued cells, range k from q_first[k]
    int32_t nq = 0;
    const int64_t* q_off = nullptr;
    const int64_t* q_first = nullptr;
    // dense outputs (no CSR): the fe / ke rows of cell c are c - ke_cell0
    int64_t ke_cell0 = 0;
    // ke layout: 0 = full row-major NE x NE (per-cell calls); 1 = the upper node-pair blocks (a <= b)
    // only: block row a holds its ND scalar rows one after another, each with the columns of nodes
    // a..NN-1 (upper_entry), NN(NN+1)/2 ND x ND blocks per cell (the gather assembly)
    int ke_upper = 0;
    // direct assembly (CSR kernels): cell c adds its node-row slab a into block row A = conn[c][a]
    // and its F_int share into R once ticket[A] equals c's rank among A's cells (crank), then
    // advances the ticket; cells are taken in ascending order from the counter `next`
    const int64_t* bptr = nullptr;       // block-row pointers [npoint + 1]
    const int16_t* cslot = nullptr;      // [cell][a][b]: column slot of node b in block row conn[a]
    const int32_t* crank = nullptr;      // [cell][a]: rank (bits 0..29), last-cell flag (bit 30)
    const uint32_t* cfirst = nullptr;    // [cell][a] bit b: first contribution to block (conn[a], conn[b])
    const int32_t* order = nullptr;      // direct assembly: the k-th dequeued position takes cell order[k]
    int32_t* ticket = nullptr;           // [npoint]: slabs of this launch already added to the row
    unsigned long long* next = nullptr;  // in-order work counter, zero at launch
    double* csr = nullptr;               // CSR values of K (DOK)
    double* ff = nullptr;                // R = F_int (DOF)
};

// Ordered-assembly tickets: acquire/release at GPU scope, so the slab a cell adds to a row is
// visible to the next cell of that row before it reads the row.
__device__ __forceinline__ int ticket_load(const int32_t* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void ticket_store(int32_t* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Polls of a row ticket before the kernel gives up (each poll sleeps up to ~1 us, so about 0.1 s):
// far beyond any legitimate wait, which is the time one earlier cell takes to finish.  A wait that
// runs out reports E_ORDER (rank 3 in the error key) and adds the slab anyway; every other wait of the
// launch sees that key within 64 polls and stops waiting too, so the kernel always ends promptly.
constexpr int ORDER_WAIT_LIMIT = 1 << 17;
__device__ __forceinline__ bool order_aborted(const unsigned long long* errkey) {
    return (*(volatile const unsigned long long*)errkey >> 56) >= 3;
}

// Next item of the in-order work counter, for the whole warp.
__device__ __forceinline__ int64_t dequeue(unsigned long long* next) {
    unsigned long long v = 0;
    if ((threadIdx.x & 31) == 0) v = atomicAdd(next, 1ull);
    return (int64_t)__shfl_sync(0xffffffffu, v, 0);
}

// Atomic add at the L2 (relaxed, GPU scope; FP64 adds round to nearest even): no load, so the
// issuing lane does not wait.  The row tickets order the adds of successive cells (each cell's
// adds come after the release store that the next cell acquires), so every entry is still summed
// in ascending cell order.
// Number of node-pair blocks (a', b'), a' <= b', in the block rows before row a (upper layout).
__host__ __device__ constexpr int upper_block(int nn, int a, int b) { return a * nn - a * (a - 1) / 2 + (b - a); }
// Upper layout of an element matrix: entry (i, j) of block (a, b), a <= b, at
// BB*upper_block(a, a) + i*(NN - a)*ND + (b - a)*ND + j (block row a, scalar rows one after another).
template <int NN, int ND>
__host__ __device__ constexpr int upper_entry(int a, int b, int i, int j) {
    return ND * ND * upper_block(NN, a, a) + i * (NN - a) * ND + (b - a) * ND + j;
}

// Asynchronous global -> shared copies (no register passes through; cp.async.wait_all, then a warp
// barrier, before the data is read).  Sizes 4, 8 and 16 bytes, both addresses aligned to the size.
template <int B>
__device__ __forceinline__ void cp_async(void* smem_dst, const void* gsrc) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (B == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
    else asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(d), "l"(gsrc), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ void red_add(double* p, double v) {
    asm volatile("red.relaxed.gpu.global.add.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}

// One ND x ND block added into the CSR values: rows pos + i*rs, columns at the block's slot; the
// lowest cell holding both nodes stores 0 + v, the later ones add to what is there.
template <int ND>
__device__ __forceinline__ void csr_add_block(double* __restrict__ csr, int64_t pos, int rs, bool first,
                                              const double (&v)[ND][ND], bool transpose) {
#pragma unroll
    for (int i = 0; i < ND; i++)
#pragma unroll
        for (int j = 0; j < ND; j++) {
            double* q = csr + pos + (int64_t)i * rs + j;
            const double x = transpose ? v[j][i] : v[i][j];
            if (first) *q = 0.0 + x;
            else red_add(q, x);
        }
}

// Poll back-off of the row-ticket waits (ns): short first, since a legitimate wait is about the
// time one earlier cell takes to write its slab.
__device__ __forceinline__ unsigned order_backoff(int spins) { return spins < 8 ? 32 : (spins < 64 ? 256 : 1024); }

// Item i of a range queue: off[k] <= i < off[k+1] maps to first[k] + (i - off[k]).
__device__ __forceinline__ int64_t queue_item(int64_t i, int n, const int64_t* __restrict__ off,
                                              const int64_t* __restrict__ first) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= i) lo = mid;
        else hi = mid;
    }
    return __ldg(first + lo) + (i - __ldg(off + lo));
}

// Which failing IP is reported.  The reference stops at the first error of its loops: the stress
// update of every cell (Elements::update_secondary_values) runs before any tangent
// (Elements::assemble_kke), and each loop goes through the cells and their IPs in ascending order
// (src/fem/elements.rs:156-181).  A failing IP offers the key
//   rank << 56 | (2^40 - 1 - cell) << 16 | (255 - ip) << 8 | code
// (rank 2: update error, 1: tangent/assembly error) and atomicMax keeps the one the reference
// would return: update errors first, then the lowest cell, then its lowest IP.
constexpr int RANK_ORDER = 3, RANK_UPDATE = 2, RANK_TANGENT = 1;
__host__ __device__ constexpr unsigned long long error_key(int rank, int64_t cell, int ip, int code) {
    return ((unsigned long long)rank << 56) | ((((1ull << 40) - 1) - (unsigned long long)cell) << 16) |
           ((unsigned long long)(255 - ip) << 8) | (unsigned long long)(code & 0xff);
}
__device__ __forceinline__ void report(const ElemArgs& A, int rank, int code, int64_t cell, int ip) {
    if (code == OK) return;
    const unsigned long long k = error_key(rank, cell, ip, code);
    atomicMax(A.errkey, k);
    if (A.prob_err && A.cell_prob) atomicMax(A.prob_err + A.cell_prob[cell], k);
}

template <int ND>
__device__ __forceinline__ double inv_jacobian(const double* J, double* Ji) {
    if (ND == 2) {
        double det = J[0] * J[3] - J[1] * J[2];
        double id = 1.0 / det;
        Ji[0] = J[3] * id;
        Ji[1] = -J[1] * id;
        Ji[2] = -J[2] * id;
        Ji[3] = J[0] * id;
        return det;
    } else {
        double c0 = J[4] * J[8] - J[5] * J[7];
        double c1 = J[5] * J[6] - J[3] * J[8];
        double c2 = J[3] * J[7] - J[4] * J[6];
        double det = J[0] * c0 + J[1] * c1 + J[2] * c2;
        double id = 1.0 / det;
        Ji[0] = c0 * id;
        Ji[1] = (J[2] * J[7] - J[1] * J[8]) * id;
        Ji[2] = (J[1] * J[5] - J[2] * J[4]) * id;
        Ji[3] = c1 * id;
        Ji[4] = (J[0] * J[8] - J[2] * J[6]) * id;
        Ji[5] = (J[2] * J[3] - J[0] * J[5]) * id;
        Ji[6] = c2 * id;
        Ji[7] = (J[1] * J[6] - J[0] * J[7]) * id;
        Ji[8] = (J[0] * J[4] - J[1] * J[3]) * id;
        return det;
    }
}

// Warps per cell.  The kernel can split a cell's node-pair triangle over two warps (2x2 register
// tiles: fewer registers per thread, more warps per SM), but for Hex20 that measured slower (4.55
// vs 4.27 ms on the 64x64x32 block: 40% more shared-memory loads per pair, and the second warp
// idles during the integration-point phase), so every kind uses one warp per cell.
__host__ __device__ constexpr int warps_per_cell(int) { return 1; }
__host__ __device__ constexpr int cells_per_block(int nn) { return WPB / warps_per_cell(nn); }

// Register tile of node pairs per lane: rows (a) x cols (b) of the upper node-pair triangle.
// The tile shapes keep the number of tiles <= 32 per warp of the cell.
template <int NN> struct TileShape;
template <int NN> __host__ __device__ constexpr int tile_count() {
    int k = 0;
    for (int i = 0; i < TileShape<NN>::NRG; i++)
        for (int j = 0; j < TileShape<NN>::NCG; j++) {
            const int jmax = (j * TileShape<NN>::CT + TileShape<NN>::CT - 1) < (NN - 1)
                                 ? (j * TileShape<NN>::CT + TileShape<NN>::CT - 1) : (NN - 1);
            if (i * TileShape<NN>::RT <= jmax) k++;
        }
    return k;
}
template <int NN> struct TileShape {
    static constexpr int RT = NN >= 13 ? 2 : 1;
    static constexpr int CT = warps_per_cell(NN) == 2 ? 2 : (NN >= 13 ? 4 : (NN >= 7 ? 2 : 1));
    static constexpr int NRG = (NN + RT - 1) / RT;
    static constexpr int NCG = (NN + CT - 1) / CT;
};

// Shared memory (doubles): block-wide dN table [m][j][32] + w[32] (+ N table [m][32] in 2D), then per cell
// X[NN*ND], dU[NN*ND], G[ng][NN*ND+1] (gradients), TC[ng][10] (alpha, gamma, beta, S), CS[ng][6],
// V (2D cells of this kernel only): per node at the current IP, V[WPC][NN][VS] = alpha g, gamma g^,
// beta h, g, h, g^, 2 (a/2)|J|w r q and q, with h = S g (+ q s_zz e_x), g^ = g (+ q e_x) and q = N/r in
// the axisymmetric idealization (double-buffered when two warps share the cell).
__host__ __device__ constexpr int node_vec_doubles(int nd) { return 5 * nd + (nd == 2 ? 4 : 0); }
__host__ __device__ constexpr int smem_table_doubles(int nn, int nd) {
    return nn * nd * 32 + 32 + (nd == 2 ? nn * 32 : 0);
}
// Direct-assembly metadata at the start of each cell area (doubles, kept even for 16-byte copies):
// per node [bptr[A], bptr[A+1], crank | cfirst << 32, A] (NM), the pending ticket releases of the
// warp's previous cell [row or -1, value] (PEND), the cell's column-slot map (CSL, int16) and its
// local nodes in ascending node id (CSORT, uint8).
__host__ __device__ constexpr int meta_doubles(int nn) {
    return 4 * nn + 2 * nn + 2 * ((nn * nn + 7) / 8) + 2 * ((nn + 15) / 16);
}
__host__ __device__ constexpr int cell_work_doubles(int nn, int nd, int ng) {
    return ng * (nn * nd + 1) + ng * 10 + ng * 6 + (nd == 3 ? 0 : warps_per_cell(nn) * nn * node_vec_doubles(nd)) +
           (ng & 1);
}
// Per cell: metadata, X and dU, then the phase work arrays; the direct assembly stages the cell's
// upper node-pair blocks over the work arrays (after dU, which then holds F_int), so the work area
// is at least that large.
__host__ __device__ constexpr int smem_cell_doubles(int nn, int nd, int ng) {
    return meta_doubles(nn) + 2 * nn * nd +
           (cell_work_doubles(nn, nd, ng) > nn * (nn + 1) / 2 * nd * nd ? cell_work_doubles(nn, nd, ng)
                                                                          : ((nn * (nn + 1) / 2 * nd * nd + 1) & ~1));
}
__host__ __device__ constexpr int smem_bytes_for(int nn, int nd, int ng, int wpb) {
    return (smem_table_doubles(nn, nd) + (wpb / warps_per_cell(nn)) * smem_cell_doubles(nn, nd, ng)) * 8;
}

template <int ND, int NN, int UPD, bool DOF, bool DOK, bool CSR>
__global__ void __launch_bounds__(WPB * 32, warps_per_cell(NN) == 2 ? 3 : (ND == 2 ? (NN >= 13 ? 2 : 4) : 1))
element_kernel(ElemArgs A) {
    static_assert(!CSR || warps_per_cell(NN) == 1, "the ordered assembly takes one warp per cell");
    constexpr int NC = 2 * ND;
    constexpr int NE = NN * ND;
    constexpr int GS = NE + 1;  // gradient row stride (odd: spreads the banks of phase-1 stores)
    using TS = TileShape<NN>;
    constexpr int RT = TS::RT, CT = TS::CT;
    constexpr int WPC = warps_per_cell(NN), CPB = WPB / WPC;
    static_assert(tile_count<NN>() <= 32 * WPC, "every node-pair tile needs a lane");
    extern __shared__ __align__(16) double smem[];
    const int ng = A.ngauss;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int cs = wid / WPC, half = wid % WPC;  // cell slot in the block, warp within the cell
    double* dNs = smem;                        // [m][j][32]
    double* ws = smem + NE * 32;               // [32]
    double* Ns = ws + 32;                      // [m][32] (2D)
    double* wbase = smem + smem_table_doubles(NN, ND) + cs * smem_cell_doubles(NN, ND, ng);
    int64_t* NM = reinterpret_cast<int64_t*>(wbase);  // [m][4] (direct assembly)
    int64_t* PEND = NM + 4 * NN;                      // [m][2] (direct assembly)
    int16_t* CSL = reinterpret_cast<int16_t*>(PEND + 2 * NN);  // [NN*NN] (direct assembly)
    uint8_t* CSORT = reinterpret_cast<uint8_t*>(CSL) + 16 * ((NN * NN + 7) / 8);  // [NN] (direct assembly)
    double* Xs = wbase + meta_doubles(NN);     // [m][d]
    double* Us = Xs + NE;                      // [m][d]
    double* G = Us + NE;                       // [p][GS]
    double* TC = G + ng * GS;                  // [p][10]
    double* CS = TC + ng * 10;                 // [p][6]
    double* V0 = CS + ng * 6;                  // [2][m][5*ND]

    // stage dN transposed (IP index fastest) so that lane p reads its IP without bank conflicts
    for (int i = threadIdx.x; i < ng * NE; i += blockDim.x) {
        const int p = i / NE, r = i % NE;
        dNs[r * 32 + p] = A.tab[i];
    }
    for (int i = threadIdx.x; i < ng; i += blockDim.x) ws[i] = A.tab[ng * NE + i];
    if (ND == 2 && A.axisym)
        for (int i = threadIdx.x; i < ng * NN; i += blockDim.x) {
            const int p = i / NN, m = i % NN;
            Ns[m * 32 + p] = A.tab[ng * NE + ng + i];
        }
    __syncthreads();

    // the warps of one cell meet at a named barrier (id 1 + cell slot)
    auto cell_sync = [&]() {
        if constexpr (WPC == 1) __syncwarp();
        else asm volatile("bar.sync %0, %1;" ::"r"(1 + cs), "r"(32 * WPC) : "memory");
    };
    // persistent: the block's cell slots walk the queue with a stride of the whole grid, or (direct
    // assembly) take the next cell from the in-order counter
    const int64_t cstride = (int64_t)gridDim.x * CPB;
    if constexpr (CSR) {
        if (lane < NN) PEND[2 * lane] = -1;  // no release pending
        __syncwarp();
    }
    for (int64_t cl = CSR ? dequeue(A.next) : (int64_t)blockIdx.x * CPB + cs; cl < A.ncell;
         cl = CSR ? dequeue(A.next) : cl + cstride) {
    cell_sync();  // the previous cell's write-out is done with the cell's shared memory
    int64_t cell = A.nq ? queue_item(cl, A.nq, A.q_off, A.q_first) : A.cell0 + cl;
    if (CSR) cell = __ldg(A.order + cell);  // processing order (a permutation within each problem)
    int mode = (UPD == UPD_NONE) ? 0 : 2;
    if (UPD == UPD_MODE) {
        mode = A.pmode[A.cell_prob[cell]];
        if (mode == 0) continue;  // inactive problem: the cell's warps skip it together
    }
    const bool do_update = (UPD == UPD_MODE) ? (mode >= 2) : (UPD != UPD_NONE);
    const bool from_backup = (UPD == UPD_BACKUP) || (UPD == UPD_MODE && mode >= 2);
    // mode 3 (batched solver, constant tangent): update and F_int, K left as it is
    const bool dok_c = DOK && !(UPD == UPD_MODE && mode == 3);
    const MatConst mc = A.mats[A.cmat ? A.cmat[cell] : 0];

    if (half == 0) {  // warp 0 of the cell: node data, integration points, F_int
    // the IP state is loaded first, so that its latency overlaps the node staging below
    const int64_t ip0 = cell * ng;
    const bool has_ip = lane < ng;
    double sig[NC], z = 0.0, lam = 0.0;
    int el = 1;
#pragma unroll
    for (int c = 0; c < NC; c++) sig[c] = 0.0;
    if (has_ip) {
        const double* ssrc = from_backup ? A.sig_src : A.sig;
        const double* zsrc = from_backup ? A.z_src : A.z;
        const double* lsrc = from_backup ? A.lam_src : A.lam;
        const uint8_t* esrc = from_backup ? A.el_src : A.el;
#pragma unroll
        for (int c = 0; c < NC; c++) sig[c] = ssrc[(int64_t)c * A.nip + ip0 + lane];
        z = zsrc[ip0 + lane];
        lam = lsrc[ip0 + lane];
        el = esrc[ip0 + lane];
    }
    if (lane < NN) {
        const int pt = A.conn[cell * NN + lane];
#pragma unroll
        for (int i = 0; i < ND; i++) {
            Xs[lane * ND + i] = A.coords[(int64_t)pt * ND + i];
            Us[lane * ND + i] = do_update ? A.ddu[(int64_t)pt * ND + i] : 0.0;
        }
    }
    __syncwarp();

    // ---------------- phase 1: lane p owns integration point p ----------------
    int err = OK, err_t = OK;  // stress-update (and geometry) error, tangent error
    if (has_ip) {
        if (UPD == UPD_MODE && mode == 1) {
            // reset_algorithmic_variables + backup_secondary_values of a new load step
            lam = 0.0;
#pragma unroll
            for (int c = 0; c < NC; c++) const_cast<double*>(A.sig_src)[(int64_t)c * A.nip + ip0 + lane] = sig[c];
            const_cast<double*>(A.z_src)[ip0 + lane] = z;
            const_cast<double*>(A.lam_src)[ip0 + lane] = 0.0;
            const_cast<uint8_t*>(A.el_src)[ip0 + lane] = (uint8_t)el;
            A.lam[ip0 + lane] = 0.0;
        }
        const int p = lane;
        double J[ND * ND];
#pragma unroll
        for (int k = 0; k < ND * ND; k++) J[k] = 0.0;
#pragma unroll
        for (int m = 0; m < NN; m++)
#pragma unroll
            for (int i = 0; i < ND; i++)
#pragma unroll
                for (int j = 0; j < ND; j++) J[i * ND + j] = fma(Xs[m * ND + i], dNs[(m * ND + j) * 32 + p], J[i * ND + j]);
        double Ji[ND * ND];
        const double det = inv_jacobian<ND>(J, Ji);
        if (!(det > 0.0)) err = E_JACOBIAN;
        // integration weight |J| w t, or |J| w r with r = sum N_m x_m (axisymmetric)
        double rad = 1.0;
        if (ND == 2 && A.axisym) {
            rad = 0.0;
#pragma unroll
            for (int m = 0; m < NN; m++) rad += Ns[m * 32 + p] * Xs[m * ND];
        }
        const double coef = det * ws[p] * ((ND == 2 && A.axisym) ? rad : A.thickness);
        double eps[NC];
#pragma unroll
        for (int c = 0; c < NC; c++) eps[c] = 0.0;
        double* Gp = G + p * GS;
#pragma unroll
        for (int m = 0; m < NN; m++) {
            double g[ND];
#pragma unroll
            for (int i = 0; i < ND; i++) {
                double v = 0.0;
#pragma unroll
                for (int j = 0; j < ND; j++) v = fma(dNs[(m * ND + j) * 32 + p], Ji[j * ND + i], v);
                g[i] = v;
                Gp[m * ND + i] = v;
            }
            if (do_update) {
                const double* u = Us + m * ND;
                eps[0] += u[0] * g[0];
                eps[1] += u[1] * g[1];
                if constexpr (ND == 2) {
                    eps[3] += SQRT2 * ((u[0] * g[1] + u[1] * g[0]) / 2.0);
                } else {
                    eps[2] += u[2] * g[2];
                    eps[3] += SQRT2 * ((u[0] * g[1] + u[1] * g[0]) / 2.0);
                    eps[4 % NC] += SQRT2 * ((u[1] * g[2 % ND] + u[2 % ND] * g[1]) / 2.0);
                    eps[5 % NC] += SQRT2 * ((u[0] * g[2 % ND] + u[2 % ND] * g[0]) / 2.0);
                }
            }
        }
        if (ND == 2 && A.axisym && do_update)  // out-of-plane strain u_r / r (calculate_strain.rs:36-48)
#pragma unroll
            for (int m = 0; m < NN; m++) eps[2] += Us[m * ND] * Ns[m * 32 + p] / rad;
        if (do_update) {
            const int st = ip_update<NC>(mc, mc.hh, sig, z, lam, el, eps);
            if (st != OK && err == OK) err = st;
        }
        if (DOF) {  // coef * sigma as a symmetric ND x ND tensor: xx, yy, xy (, zz, yz, xz)
            double* c6 = CS + p * 6;
            c6[0] = coef * sig[0];
            c6[1] = coef * sig[1];
            c6[2] = coef * sig[3] * INV_SQRT2;
            if constexpr (ND == 2) {
                c6[3] = coef * sig[2];  // hoop stress (axisymmetric)
                c6[4] = rad;
            }
            if constexpr (ND == 3) {
                c6[3] = coef * sig[2];
                c6[4] = coef * sig[4 % NC] * INV_SQRT2;
                c6[5] = coef * sig[5 % NC] * INV_SQRT2;
            }
        }
        if (dok_c) {
            double a, b, s[NC];
            err_t = tangent_coefs<NC>(mc, mc.hh, sig, lam, el, a, b, s);
            double* t = TC + p * 10;
            t[0] = coef * 0.5 * a;
            // volumetric coefficient: K - a/3 (= Lame lambda when elastic); plane stress: lambda*
            t[1] = coef * ((ND == 2 && mc.plane_stress) ? mc.ps12 : (mc.kk - a / 3.0));
            t[2] = coef * b;
            t[3] = s[0];
            t[4] = s[1];
            t[5] = s[3] * INV_SQRT2;
            if constexpr (ND == 2) {
                t[6] = s[2];  // deviatoric s_zz (axisymmetric hoop row)
                t[9] = rad;
            }
            if constexpr (ND == 3) {
                t[6] = s[2];
                t[7] = s[4 % NC] * INV_SQRT2;
                t[8] = s[5 % NC] * INV_SQRT2;
            }
        }
    }
    // first failing IP of the cell (lowest p): an update error if any, else a tangent error
    {
        const unsigned bad = __ballot_sync(FULL, err != OK);
        const unsigned bad_t = __ballot_sync(FULL, err_t != OK);
        if (bad) {
            const int p = __ffs(bad) - 1;
            const int code = __shfl_sync(FULL, err, p);
            if (lane == 0) report(A, do_update ? RANK_UPDATE : RANK_TANGENT, code, cell, p);
        } else if (bad_t) {
            const int p = __ffs(bad_t) - 1;
            const int code = __shfl_sync(FULL, err_t, p);
            if (lane == 0) report(A, RANK_TANGENT, code, cell, p);
        }
    }
    if (do_update && has_ip) {
#pragma unroll
        for (int c = 0; c < NC; c++) A.sig[(int64_t)c * A.nip + ip0 + lane] = sig[c];
        A.z[ip0 + lane] = z;
        A.lam[ip0 + lane] = lam;
        A.el[ip0 + lane] = (uint8_t)el;
    }
    __syncwarp();

    // ---------------- F_int: lane m owns node m ----------------
    if (DOF && lane < NN) {
        double f[ND];
#pragma unroll
        for (int i = 0; i < ND; i++) f[i] = 0.0;
        for (int p = 0; p < ng; p++) {
            const double* c6 = CS + p * 6;
            const double* g = G + p * GS + lane * ND;
            if constexpr (ND == 2) {
                f[0] += c6[0] * g[0] + c6[2] * g[1];
                f[1] += c6[2] * g[0] + c6[1] * g[1];
                if (A.axisym) f[0] += c6[3] * Ns[lane * 32 + p] / c6[4];
            } else {
                f[0] += c6[0] * g[0] + c6[2] * g[1] + c6[5 % 6] * g[2 % ND];
                f[1] += c6[2] * g[0] + c6[1] * g[1] + c6[4 % 6] * g[2 % ND];
                f[2 % ND] += c6[5 % 6] * g[0] + c6[4 % 6] * g[1] + c6[3 % 6] * g[2 % ND];
            }
        }
        // direct assembly: kept in the cell's dU slot (free after phase 1) until the scatter
#pragma unroll
        for (int i = 0; i < ND; i++) {
            if (CSR) Us[lane * ND + i] = f[i];
            else A.fe[((cell - A.ke_cell0) * NN + lane) * ND + i] = f[i];
        }
    }

    }  // warp 0
    cell_sync();  // G and TC are visible to every warp of the cell
    if constexpr (CSR) {
        if (DOF || DOK) {  // the scatter's row data and slot map, copied while the node pairs are computed
            if (lane < NN) {
                const int64_t pt = A.conn[cell * NN + lane];
                int64_t* nm = NM + 4 * lane;
                cp_async<8>(nm, A.bptr + pt);
                cp_async<8>(nm + 1, A.bptr + pt + 1);
                cp_async<4>(nm + 2, A.crank + cell * NN + lane);
                cp_async<4>(reinterpret_cast<int32_t*>(nm + 2) + 1, A.cfirst + cell * NN + lane);
                nm[3] = pt;
            }
            constexpr int CB = NN * NN * 2;  // bytes of the cell's slot map
            const char* src = reinterpret_cast<const char*>(A.cslot + cell * (int64_t)(NN * NN));
            char* dst = reinterpret_cast<char*>(CSL);
            if constexpr (CB % 16 == 0) {
                for (int k = lane; k < CB / 16; k += 32) cp_async<16>(dst + 16 * k, src + 16 * k);
            } else if constexpr (CB % 8 == 0) {
                for (int k = lane; k < CB / 8; k += 32) cp_async<8>(dst + 8 * k, src + 8 * k);
            } else {  // a map whose cell offset is not 4-byte aligned (Tri15): plain loads
                for (int k = lane; k < NN * NN; k += 32) CSL[k] = A.cslot[cell * (int64_t)(NN * NN) + k];
            }
        }
    }

    // ---------------- phase 2: lane owns a tile of node-pair blocks ----------------
    int ti = -1, tj = -1;
    double acc[RT][CT][ND][ND];
    if (dok_c) {
        // tile number lane + 32*half: (i, j) with i*RT <= min(j*CT + CT - 1, NN - 1), row-major
        {
            const int me = lane + 32 * half;
            int k = 0;
            for (int i = 0; i < TS::NRG; i++)
                for (int j = 0; j < TS::NCG; j++) {
                    const int jmax = min(j * CT + CT - 1, NN - 1);
                    if (i * RT <= jmax) {
                        if (k == me) { ti = i; tj = j; }
                        k++;
                    }
                }
        }
        const int a0 = ti * RT, b0 = tj * CT;
#pragma unroll
        for (int r = 0; r < RT; r++)
#pragma unroll
            for (int c = 0; c < CT; c++)
#pragma unroll
                for (int i = 0; i < ND; i++)
#pragma unroll
                    for (int j = 0; j < ND; j++) acc[r][c][i][j] = 0.0;
        if constexpr (ND == 3) {
        // Two passes, each entry with a fixed operation order.  With X_ab = sum_p alpha_p g_a g_b^T
        // (alpha = w|J| a/2) the blocks are
        //   K_ab = X_ab^T + tr(X_ab) 1 + c X_ab + sum over plastic p of (kappa_p g_a g_b^T + beta_p h_a h_b^T)
        // with c = lambda/G and kappa_p = gamma_p - c alpha_p (gamma = w|J|(K - a/3)): an elastic
        // point has a = 2G, so gamma = c alpha there and it adds to X only (9 FMA per node pair,
        // against 27 at a plastic point).  Pass A needs no staging: alpha comes from TC and g from
        // the gradients of phase 1.
        static_assert(WPC == 1, "the 3D node-pair phase takes one warp per cell");
        const double cvol = (mc.kk - 2.0 * mc.gg / 3.0) / mc.gg;
        if (ti >= 0) {
            for (int p = 0; p < ng; p++) {
                const double al = TC[p * 10];
                const double* g = G + p * GS;
                double ar[RT][3];
#pragma unroll
                for (int r = 0; r < RT; r++)
#pragma unroll
                    for (int i = 0; i < 3; i++) ar[r][i] = al * g[min(a0 + r, NN - 1) * 3 + i];
#pragma unroll
                for (int c = 0; c < CT; c++) {
                    double gb[3];
#pragma unroll
                    for (int j = 0; j < 3; j++) gb[j] = g[min(b0 + c, NN - 1) * 3 + j];
#pragma unroll
                    for (int r = 0; r < RT; r++)
#pragma unroll
                        for (int i = 0; i < 3; i++)
#pragma unroll
                            for (int j = 0; j < 3; j++) acc[r][c][i][j] = fma(ar[r][i], gb[j], acc[r][c][i][j]);
                }
            }
#pragma unroll
            for (int r = 0; r < RT; r++)
#pragma unroll
                for (int c = 0; c < CT; c++) {
                    double x[3][3];
#pragma unroll
                    for (int i = 0; i < 3; i++)
#pragma unroll
                        for (int j = 0; j < 3; j++) x[i][j] = acc[r][c][i][j];
                    const double tr = x[0][0] + x[1][1] + x[2][2];
#pragma unroll
                    for (int i = 0; i < 3; i++)
#pragma unroll
                        for (int j = 0; j < 3; j++) {
                            const double v = fma(cvol, x[i][j], x[j][i]);
                            acc[r][c][i][j] = (i == j) ? v + tr : v;
                        }
                }
        }
        // pass B, plastic points only: every lane forms kappa g, beta h and h = S g of its own row and
        // column nodes (the same operations the node would stage), so the points need no staging and
        // no barrier and follow each other without a wait
        if (ti >= 0) {
            for (int p = 0; p < ng; p++) {
                const double* t = TC + p * 10;
                const double be = t[2];
                if (be == 0.0) continue;  // elastic point: same value on every lane, uniform branch
                const double kap = t[1] - cvol * t[0];
                double S[3][3];
                S[0][0] = t[3];
                S[1][1] = t[4];
                S[2][2] = t[6];
                S[0][1] = S[1][0] = t[5];
                S[1][2] = S[2][1] = t[7];
                S[0][2] = S[2][0] = t[8];
                const double* g = G + p * GS;
                double kr[RT][3], hr[RT][3];
#pragma unroll
                for (int r = 0; r < RT; r++) {
                    const double* ga = g + min(a0 + r, NN - 1) * 3;
                    const double gv[3] = {ga[0], ga[1], ga[2]};
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        double h = 0.0;
#pragma unroll
                        for (int j = 0; j < 3; j++) h = fma(S[i][j], gv[j], h);
                        kr[r][i] = kap * gv[i];
                        hr[r][i] = be * h;
                    }
                }
#pragma unroll
                for (int c = 0; c < CT; c++) {
                    const double* gbp = g + min(b0 + c, NN - 1) * 3;
                    const double gb[3] = {gbp[0], gbp[1], gbp[2]};
                    double hb[3];
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        double h = 0.0;
#pragma unroll
                        for (int j = 0; j < 3; j++) h = fma(S[i][j], gb[j], h);
                        hb[i] = h;
                    }
#pragma unroll
                    for (int r = 0; r < RT; r++)
#pragma unroll
                        for (int i = 0; i < 3; i++)
#pragma unroll
                            for (int j = 0; j < 3; j++) {
                                acc[r][c][i][j] = fma(kr[r][i], gb[j], acc[r][c][i][j]);
                                acc[r][c][i][j] = fma(hr[r][i], hb[j], acc[r][c][i][j]);
                            }
                }
            }
        }
        } else {
        constexpr int VS = node_vec_doubles(ND);
        for (int p = 0; p < ng; p++) {
            const double* t = TC + p * 10;
            const bool plastic = t[2] != 0.0;  // beta: same value on every lane, uniform branch
            // two warps: double buffer, one barrier per IP; one warp: every lane is done with the
            // previous IP's vectors before the node lanes overwrite them
            double* V = V0 + (WPC == 2 ? (p & 1) * NN * VS : 0);
            if constexpr (WPC == 1) __syncwarp();
            // node lanes of warp 0: the scaled gradients of their node at this IP
            if (half == 0 && lane < NN) {
                const double al = t[0], ga = t[1], be = t[2];
                double S[ND][ND];
                S[0][0] = t[3];
                S[1][1] = t[4];
                S[0][1] = S[1][0] = t[5];
                if constexpr (ND == 3) {
                    S[2 % ND][2 % ND] = t[6];
                    S[1][2 % ND] = S[2 % ND][1] = t[7];
                    S[0][2 % ND] = S[2 % ND][0] = t[8];
                }
                const double* g = G + p * GS + lane * ND;
                double* v = V + lane * VS;
                double gv[ND], gh[ND];  // gradient and volumetric row B^T I (with the hoop term)
#pragma unroll
                for (int i = 0; i < ND; i++) gh[i] = gv[i] = g[i];
                double q = 0.0;  // N/r of this node (axisymmetric)
                if (ND == 2 && A.axisym) {
                    q = Ns[lane * 32 + p] / t[9];
                    gh[0] = gv[0] + q;
                }
#pragma unroll
                for (int i = 0; i < ND; i++) {
                    double h = 0.0;
                    if (plastic) {
#pragma unroll
                        for (int j = 0; j < ND; j++) h = fma(S[i][j], gv[j], h);
                        if (ND == 2 && A.axisym && i == 0) h = fma(q, t[6], h);
                    }
                    v[i] = al * gv[i];
                    v[ND + i] = ga * gh[i];
                    v[2 * ND + i] = be * h;
                    v[3 * ND + i] = gv[i];
                    v[4 * ND + i] = h;
                }
                if constexpr (ND == 2) {
                    v[5 * ND] = gh[0];
                    v[5 * ND + 1] = gh[1];
                    v[5 * ND + 2] = 2.0 * al * q;
                    v[5 * ND + 3] = q;
                }
            }
            cell_sync();
            if (ti < 0) continue;
            double Ar[RT][ND], Cr[RT][ND], Hr[RT][ND], Qr[RT];
#pragma unroll
            for (int r = 0; r < RT; r++) {
                const double* v = V + min(a0 + r, NN - 1) * VS;
#pragma unroll
                for (int i = 0; i < ND; i++) {
                    Ar[r][i] = v[i];
                    Cr[r][i] = v[ND + i];
                    Hr[r][i] = v[2 * ND + i];
                }
                Qr[r] = (ND == 2) ? v[(5 * ND + 2) % VS] : 0.0;
            }
#pragma unroll
            for (int c = 0; c < CT; c++) {
                const double* v = V + min(b0 + c, NN - 1) * VS;
                double gb[ND], hb[ND], gc[ND];  // g, h and the volumetric row of the column node
#pragma unroll
                for (int i = 0; i < ND; i++) {
                    gb[i] = v[3 * ND + i];
                    hb[i] = v[4 * ND + i];
                    gc[i] = (ND == 2) ? v[(5 * ND + i) % VS] : gb[i];
                }
                const double qb = (ND == 2) ? v[(5 * ND + 3) % VS] : 0.0;
                double dot[RT];
#pragma unroll
                for (int r = 0; r < RT; r++) {
                    dot[r] = 0.0;
#pragma unroll
                    for (int k = 0; k < ND; k++) dot[r] = fma(Ar[r][k], gb[k], dot[r]);
                }
                // term by term over the tile column (each entry keeps its own operation order)
#pragma unroll
                for (int r = 0; r < RT; r++)
#pragma unroll
                    for (int i = 0; i < ND; i++)
#pragma unroll
                        for (int j = 0; j < ND; j++) acc[r][c][i][j] = fma(Ar[r][j], gb[i], acc[r][c][i][j]);
#pragma unroll
                for (int r = 0; r < RT; r++)
#pragma unroll
                    for (int i = 0; i < ND; i++)
#pragma unroll
                        for (int j = 0; j < ND; j++) acc[r][c][i][j] = fma(Cr[r][i], gc[j], acc[r][c][i][j]);
                if (plastic) {
#pragma unroll
                    for (int r = 0; r < RT; r++)
#pragma unroll
                        for (int i = 0; i < ND; i++)
#pragma unroll
                            for (int j = 0; j < ND; j++) acc[r][c][i][j] = fma(Hr[r][i], hb[j], acc[r][c][i][j]);
                }
#pragma unroll
                for (int r = 0; r < RT; r++)
#pragma unroll
                    for (int i = 0; i < ND; i++) acc[r][c][i][i] += dot[r];
                if (ND == 2 && A.axisym)  // hoop row: a (N_a/r)(N_b/r) on the radial-radial entry
#pragma unroll
                    for (int r = 0; r < RT; r++) acc[r][c][0][0] = fma(Qr[r], qb, acc[r][c][0][0]);
            }
        }
        }  // ND
        if constexpr (CSR) {  // direct assembly: stage the upper blocks after dU for the scatter
            double* KS = Us + NE;
            if (ti >= 0) {
#pragma unroll
                for (int r = 0; r < RT; r++)
#pragma unroll
                    for (int c = 0; c < CT; c++) {
                        const int a = a0 + r, b = b0 + c;
                        if (a < NN && b < NN && a <= b) {
#pragma unroll
                            for (int i = 0; i < ND; i++)
#pragma unroll
                                for (int j = 0; j < ND; j++) KS[upper_entry<NN, ND>(a, b, i, j)] = acc[r][c][i][j];
                        }
                    }
            }
        }
        // dense output: write K_e (row-major NE x NE) through the warp's shared memory, RS node rows at a time:
        // each lane drops its blocks (a, b) and mirrors (b, a) into the staged rows, then the warp
        // copies the rows out with contiguous stores
        if constexpr (!CSR) {
        if (A.ke_upper) {
            // upper blocks only: block rows [r0, r0 + RS) are the contiguous range [u(r0, r0), u(r0 + RS, .))
            constexpr int NU = NN * (NN + 1) / 2, BB = ND * ND;
            const int RS = max(1, min(NN, smem_cell_doubles(NN, ND, ng) / (NN * BB)));
            double* stage = wbase;
            double* kc = A.ke + (cell - A.ke_cell0) * (int64_t)(NU * BB);
            for (int r0 = 0; r0 < NN; r0 += RS) {
                const int r1 = min(NN, r0 + RS);
                const int u0 = upper_block(NN, r0, r0), u1 = (r1 < NN) ? upper_block(NN, r1, r1) : NU;
                cell_sync();
                if (ti >= 0) {
#pragma unroll
                    for (int r = 0; r < RT; r++)
#pragma unroll
                        for (int c = 0; c < CT; c++) {
                            const int a = a0 + r, b = b0 + c;
                            if (a < NN && b < NN && a <= b && a >= r0 && a < r1) {
#pragma unroll
                                for (int i = 0; i < ND; i++)
#pragma unroll
                                    for (int j = 0; j < ND; j++)
                                        stage[upper_entry<NN, ND>(a, b, i, j) - u0 * BB] = acc[r][c][i][j];
                            }
                        }
                }
                cell_sync();
                const int n = (u1 - u0) * BB;
                double* dst = kc + (int64_t)u0 * BB;
                for (int t = lane + 32 * half; t < n; t += 32 * WPC) dst[t] = stage[t];
            }
        } else {
        const int RS = min(NN, smem_cell_doubles(NN, ND, ng) / (ND * NE));
        double* stage = wbase;
        double* kc = A.ke + (cell - A.ke_cell0) * (int64_t)(NE * NE);
        for (int r0 = 0; r0 < NN; r0 += RS) {
            cell_sync();
            if (ti >= 0) {
#pragma unroll
                for (int r = 0; r < RT; r++)
#pragma unroll
                    for (int c = 0; c < CT; c++) {
                        const int a = a0 + r, b = b0 + c;
                        if (a < NN && b < NN && a <= b) {
                            if (a >= r0 && a < r0 + RS) {
#pragma unroll
                                for (int i = 0; i < ND; i++)
#pragma unroll
                                    for (int j = 0; j < ND; j++)
                                        stage[((a - r0) * ND + i) * NE + b * ND + j] = acc[r][c][i][j];
                            }
                            if (a != b && b >= r0 && b < r0 + RS) {
#pragma unroll
                                for (int j = 0; j < ND; j++)
#pragma unroll
                                    for (int i = 0; i < ND; i++)
                                        stage[((b - r0) * ND + j) * NE + a * ND + i] = acc[r][c][i][j];
                            }
                        }
                    }
            }
            cell_sync();
            const int n = min(RS, NN - r0) * ND * NE;
            double* dst = kc + (int64_t)r0 * ND * NE;
            for (int t = lane + 32 * half; t < n; t += 32 * WPC) dst[t] = stage[t];
        }
        }  // full layout
        }  // dense output
    }
    // ---------------- direct assembly: ordered scatter into the CSR values and R ----------------
    // The lanes stage the cell's upper node-pair blocks in shared memory (over the phase work
    // arrays, after dU, which holds F_int).  Node lane m then takes row A = conn[m] once ticket[A]
    // equals this cell's rank among A's cells; for every ready row the whole warp writes the row's
    // values -- block (m, b) for every local node b, read transposed from block (b, m) when b < m --
    // with the nodes taken in ascending node id, which is ascending column slot in every row, so
    // consecutive lanes write consecutive CSR positions.  Node lane m then advances ticket[A] (the
    // last cell of A puts it back to 0 for the next launch).  Rows become ready in rounds, so this
    // cell never waits for a row it could already write.
    if constexpr (CSR) {
        if (DOF || DOK) {
            const double* KS = Us + NE;  // the cell's upper blocks, staged at the end of phase 2
            cp_async_wait_all();
            __syncwarp();  // the staged blocks and every lane's copies are visible
            // release the rows the warp's previous cell left pending before anything can wait here:
            // a warp never waits while it holds a release
            if (lane < NN && PEND[2 * lane] >= 0) {
                ticket_store(A.ticket + PEND[2 * lane], (int)PEND[2 * lane + 1]);
                PEND[2 * lane] = -1;
            }
            int64_t rowA = INT64_MAX, pos_m = 0;
            int rs_m = 0, rank_m = 0;
            bool last_m = false, todo = false;
            if (lane < NN) {
                const int64_t* nm = NM + 4 * lane;
                rowA = nm[3];
                const int64_t r0 = nm[0], r1 = nm[1];
                pos_m = (int64_t)ND * ND * r0;
                rs_m = ND * (int)(r1 - r0);
                const int32_t cr = reinterpret_cast<const int32_t*>(nm + 2)[0];
                rank_m = cr & CRANK_MASK;
                last_m = (cr & CRANK_LAST) != 0;
                todo = true;
            }
            {  // the cell's local nodes in ascending node id
                int rk = 0;
#pragma unroll
                for (int q = 0; q < NN; q++) rk += __shfl_sync(FULL, rowA, q) < rowA;
                if (lane < NN) CSORT[rk] = (uint8_t)lane;
            }
            __syncwarp();
            int spins = 0;
            while (true) {
                const unsigned todo_mask = __ballot_sync(FULL, todo);
                if (!todo_mask) break;
                bool ready = todo && ticket_load(A.ticket + rowA) == rank_m;
                unsigned rmask = __ballot_sync(FULL, ready);
                if (!rmask) {
                    ++spins;
                    const bool give_up = __shfl_sync(FULL, spins >= ORDER_WAIT_LIMIT || ((spins & 63) == 0 && order_aborted(A.errkey)), 0);
                    if (!give_up) {
                        __nanosleep(order_backoff(spins));
                        continue;
                    }
                    if (lane == 0) report(A, RANK_ORDER, E_ORDER, cell, 0);
                    ready = todo;
                    rmask = todo_mask;
                }
                __syncwarp();  // the node lanes' acquires order every lane's writes after the earlier cells'
                if (DOF && ready) {
#pragma unroll
                    for (int i = 0; i < ND; i++) {
                        double* q = A.ff + rowA * ND + i;
                        if (rank_m == 0) *q = 0.0 + Us[lane * ND + i];
                        else red_add(q, Us[lane * ND + i]);
                    }
                }
                if (dok_c) {
                    for (unsigned rows = rmask; rows; rows &= rows - 1) {  // the ready rows, one by one
                        const int a = __ffs(rows) - 1;
                        const int64_t pa = __shfl_sync(FULL, pos_m, a);
                        const int rsa = __shfl_sync(FULL, rs_m, a);
                        // block (A, B) and its mirror get their first contribution from the first cell
                        // holding both nodes (cfirst bit b of row a)
                        const uint32_t fa = reinterpret_cast<const uint32_t*>(NM + 4 * a + 2)[1];
                        for (int e = lane; e < ND * NN * ND; e += 32) {
                            const int i = e / (NN * ND), k = (e - i * NN * ND) / ND, j = e - i * NN * ND - k * ND;
                            const int b = CSORT[k];
                            const double v = (a <= b) ? KS[upper_entry<NN, ND>(a, b, i, j)] : KS[upper_entry<NN, ND>(b, a, j, i)];
                            double* q = A.csr + pa + (int64_t)i * rsa + ND * (int64_t)CSL[a * NN + b] + j;
                            if ((fa >> b) & 1u) *q = 0.0 + v;
                            else red_add(q, v);
                        }
                    }
                }
                __syncwarp();  // every lane's writes precede the node lanes' (cumulative) release stores
                // the rows of the last round are released at the warp's next scatter (or its exit),
                // when these writes are long done, so the release does not wait for them here
                const bool final = rmask == todo_mask;
                if (ready) {
                    if (final) {
                        PEND[2 * lane] = rowA;
                        PEND[2 * lane + 1] = last_m ? 0 : rank_m + 1;
                    } else {
                        ticket_store(A.ticket + rowA, last_m ? 0 : rank_m + 1);
                    }
                }
                todo = todo && !ready;
            }
        }
    }
    }  // cells
    if constexpr (CSR) {  // the last cell's pending releases
        if (lane < NN && PEND[2 * lane] >= 0) ticket_store(A.ticket + PEND[2 * lane], (int)PEND[2 * lane + 1]);
    }
}

// ------------------------------------------------------------------------------------------------
// 2D kernel: several cells per warp, LPC lanes per cell.
//
// The 2D cells have at most 9 nodes and, in the rules used here, at most 16 integration points,
// so element_kernel (one warp per cell) keeps most lanes idle.  Here slot h of a warp owns cell
// CPW*(group) + h, CPW = 32/LPC: lane p < ngauss of the slot owns integration point p (phase 1, as
// in element_kernel), lane m < nnode owns node m (F_int), and in phase 2 lane t owns tile t of the
// upper node-pair triangle (2x2 node pairs for Tri6/Qua8/Qua9, single pairs for Tri3/Qua4).  Qua8
// with 9 points runs three cells of 10 lanes per warp (30 of 32 lanes hold a tile in phase 2).
// Phase 1 also forms, per integration point and node, h = S g (+ q s_zz e_x) and q = N/r, so
// phase 2 reads its operands from shared memory with no per-point staging or barrier.  Every
// entry of K_e and f_e takes the same operations in the same order as in element_kernel, so the
// kernels give the same bits.  A slot without a cell (ragged end, inactive problem) repeats the
// group's first cell and writes nothing: all slots run the same loop trips, so the warp-wide syncs
// below are always reached by all 32 lanes.
constexpr int WPB2 = 4;      // warps per block
constexpr int NG2_MAX = 16;  // integration points per cell that the 2D layouts hold

template <int NN> struct Tile2 {
    static constexpr int T = NN * (NN + 1) / 2 > 16 ? 2 : 1;  // tile side in nodes
    static constexpr int NG = (NN + T - 1) / T;                // node groups
    static constexpr int NT = NG * (NG + 1) / 2;               // tiles of the upper triangle
};

// Shared memory (doubles): table dN[m*2+j][16], w[16], N[m][16]; then per cell X[NE], dU[NE],
// G[ng][NE+2], H[ng][NE+2], Q[ng][NN] (+1 to an even count), TC[ng][4] (alpha, gamma, beta),
// CS[ng][6]; the cell area
// also stages K_e (NE x NE) for the write-out.
__host__ __device__ constexpr int table2_doubles(int nn) { return 2 * nn * 16 + 16 + nn * 16; }
// (every array starts on a 16-byte boundary: Q is padded to an even count)
__host__ __device__ constexpr int cell2_doubles(int nn, int ng) {
    return ((4 * nn + 2 * ng * (2 * nn + 2) + ((ng * nn + 1) & ~1) + 10 * ng > 4 * nn * nn
                 ? 4 * nn + 2 * ng * (2 * nn + 2) + ((ng * nn + 1) & ~1) + 10 * ng
                 : 4 * nn * nn) + 1) & ~1;
}
// The direct-assembly metadata (after all cell areas) only for the kernels that assemble directly.
__host__ __device__ constexpr int smem2_bytes(int nn, int ng, int cpw, bool csr) {
    return (table2_doubles(nn) + cpw * WPB2 * (cell2_doubles(nn, ng) + (csr ? meta_doubles(nn) : 0))) * 8;
}

// Lanes per cell of the packed layout: enough for every node, every node-pair tile and (checked at
// launch) every integration point.  It is used when it packs three or more cells into a warp
// (Tri3, Tri6, Qua4, Qua8: 3 to 5 cells); otherwise, and for rules with more points than lanes,
// the kernel runs with 16 lanes (two cells) per warp.
template <int NN> __host__ __device__ constexpr int lanes_packed() {
    return Tile2<NN>::NT > NN ? Tile2<NN>::NT : NN;
}
template <int NN> __host__ __device__ constexpr bool packed_layout() { return 32 / lanes_packed<NN>() >= 3; }
// Whether a 2D kind fits the several-cells-per-warp layout (at most 16 lanes per cell); larger
// cells (Tri15: 36 node-pair tiles) run in element_kernel with one warp per cell.
template <int NN> __host__ __device__ constexpr bool fits_2d() { return Tile2<NN>::NT <= 16 && NN <= 16; }

template <int NN, int LPC, int UPD, bool DOF, bool DOK, bool CSR>
__global__ void __launch_bounds__(WPB2 * 32, 4) element2d_kernel(ElemArgs A) {
    constexpr int NE = 2 * NN, GS = NE + 2;
    constexpr int CPW = 32 / LPC;  // cells per warp
    using TL = Tile2<NN>;
    constexpr int T = TL::T;
    static_assert(TL::NT <= LPC && NN <= LPC && LPC <= 16, "every node and node-pair tile needs a lane of the cell");
    extern __shared__ __align__(16) double smem2[];
    const int ng = A.ngauss;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    // cell slot of the lane in its warp and lane within the cell; the lanes past CPW*LPC join the
    // last slot with hl >= LPC, so they own no node, point or tile
    const int hh = min(lane / LPC, CPW - 1), hl = lane - hh * LPC;
    const int cd = cell2_doubles(NN, ng);
    double* dNs = smem2;          // [m*2+j][16]
    double* ws = dNs + NE * 16;   // [16]
    double* Ns = ws + 16;         // [m][16]
    double* Xs = smem2 + table2_doubles(NN) + (CPW * wid + hh) * cd;
    // direct assembly: the slot's row data, pending releases and slot map (as in element_kernel)
    int64_t* NM = CSR ? reinterpret_cast<int64_t*>(smem2 + table2_doubles(NN) + CPW * WPB2 * cd +
                                                   (CPW * wid + hh) * meta_doubles(NN))
                      : reinterpret_cast<int64_t*>(smem2);  // not used without the direct assembly
    int64_t* PEND = NM + 4 * NN;
    int16_t* CSL = reinterpret_cast<int16_t*>(PEND + 2 * NN);
    uint8_t* CSORT = reinterpret_cast<uint8_t*>(CSL) + 16 * ((NN * NN + 7) / 8);
    double* Us = Xs + NE;
    double* G = Us + NE;       // [p][GS]
    double* H = G + ng * GS;   // [p][GS]
    double* Q = H + ng * GS;   // [p][NN]
    double* TC = Q + ((ng * NN + 1) & ~1);  // [p][4]
    double* CS = TC + ng * 4;  // [p][6]

    for (int i = threadIdx.x; i < ng * NE; i += blockDim.x) {
        const int p = i / NE, r = i % NE;
        dNs[r * 16 + p] = A.tab[i];
    }
    for (int i = threadIdx.x; i < ng; i += blockDim.x) ws[i] = A.tab[ng * NE + i];
    if (A.axisym)
        for (int i = threadIdx.x; i < ng * NN; i += blockDim.x) {
            const int p = i / NN, m = i % NN;
            Ns[m * 16 + p] = A.tab[ng * NE + ng + i];
        }
    __syncthreads();

    // this lane's tile (ti <= tj), row-major over the upper triangle of node groups
    int ti = -1, tj = -1;
    {
        int k = 0;
        for (int i = 0; i < TL::NG; i++)
            for (int j = i; j < TL::NG; j++) {
                if (k == hl) {
                    ti = i;
                    tj = j;
                }
                k++;
            }
    }

    if constexpr (CSR) {
        if (hl < NN) PEND[2 * hl] = -1;  // no release pending
        __syncwarp();
    }
    const int64_t ngroup = (A.ncell + CPW - 1) / CPW;
    // groups of CPW consecutive cells: grid-strided, or (direct assembly) from the in-order counter
    for (int64_t pr = CSR ? dequeue(A.next) : (int64_t)blockIdx.x * WPB2 + wid; pr < ngroup;
         pr = CSR ? dequeue(A.next) : pr + (int64_t)gridDim.x * WPB2) {
        __syncwarp();  // the previous group's write-out is done with the cells' shared memory
        // every lane looks at all cells of the group, so the choices below agree across the warp;
        // a slot without a cell repeats the group's first cell and writes nothing
        bool active = false, any = false;
        int64_t cell = 0, cell_first = 0;
        int mode = 0, mode_first = 0;
#pragma unroll
        for (int k = 0; k < CPW; k++) {
            const int64_t cl = (int64_t)CPW * pr + k;
            bool on = cl < A.ncell;
            int64_t ck = 0;
            int mk = (UPD == UPD_NONE) ? 0 : 2;
            if (on) ck = A.nq ? queue_item(cl, A.nq, A.q_off, A.q_first) : A.cell0 + cl;
            if (CSR && on) ck = __ldg(A.order + ck);  // processing order
            if (UPD == UPD_MODE && on) {  // cells of inactive problems are left out
                mk = A.pmode[A.cell_prob[ck]];
                on = mk != 0;
            }
            if (on && !any) {
                any = true;
                cell_first = ck;
                mode_first = mk;
            }
            if (k == hh) {
                active = on;
                cell = ck;
                mode = mk;
            }
        }
        if (!any) continue;
        if (!active) {
            cell = cell_first;
            mode = mode_first;
        }
        const bool do_update = (UPD == UPD_MODE) ? (mode >= 2) : (UPD != UPD_NONE);
        const bool from_backup = (UPD == UPD_BACKUP) || (UPD == UPD_MODE && mode >= 2);
        // mode 3 (batched solver, constant tangent): update and F_int, K left as it is
        const bool dok_c = DOK && active && !(UPD == UPD_MODE && mode == 3);
        const MatConst mc = A.mats[A.cmat ? A.cmat[cell] : 0];

        // the IP state first, so that its latency overlaps the node staging
        const int64_t ip0 = cell * ng;
        const bool has_ip = hl < ng;
        double sig[4], z = 0.0, lam = 0.0;
        int el = 1;
#pragma unroll
        for (int c = 0; c < 4; c++) sig[c] = 0.0;
        if (has_ip) {
            const double* ssrc = from_backup ? A.sig_src : A.sig;
            const double* zsrc = from_backup ? A.z_src : A.z;
            const double* lsrc = from_backup ? A.lam_src : A.lam;
            const uint8_t* esrc = from_backup ? A.el_src : A.el;
#pragma unroll
            for (int c = 0; c < 4; c++) sig[c] = ssrc[(int64_t)c * A.nip + ip0 + hl];
            z = zsrc[ip0 + hl];
            lam = lsrc[ip0 + hl];
            el = esrc[ip0 + hl];
        }
        if (hl < NN) {
            const int pt = A.conn[cell * NN + hl];
#pragma unroll
            for (int i = 0; i < 2; i++) {
                Xs[hl * 2 + i] = A.coords[(int64_t)pt * 2 + i];
                Us[hl * 2 + i] = do_update ? A.ddu[(int64_t)pt * 2 + i] : 0.0;
            }
        }
        __syncwarp();

        // ---------------- phase 1: lane p of the half owns integration point p ----------------
        int err = OK, err_t = OK;  // stress-update (and geometry) error, tangent error
        if (has_ip) {
            if (UPD == UPD_MODE && mode == 1) {
                // reset_algorithmic_variables + backup_secondary_values of a new load step
                lam = 0.0;
                if (active) {
#pragma unroll
                    for (int c = 0; c < 4; c++) const_cast<double*>(A.sig_src)[(int64_t)c * A.nip + ip0 + hl] = sig[c];
                    const_cast<double*>(A.z_src)[ip0 + hl] = z;
                    const_cast<double*>(A.lam_src)[ip0 + hl] = 0.0;
                    const_cast<uint8_t*>(A.el_src)[ip0 + hl] = (uint8_t)el;
                    A.lam[ip0 + hl] = 0.0;
                }
            }
            const int p = hl;
            double J[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int m = 0; m < NN; m++)
#pragma unroll
                for (int i = 0; i < 2; i++)
#pragma unroll
                    for (int j = 0; j < 2; j++) J[i * 2 + j] = fma(Xs[m * 2 + i], dNs[(m * 2 + j) * 16 + p], J[i * 2 + j]);
            double Ji[4];
            const double det = inv_jacobian<2>(J, Ji);
            if (!(det > 0.0)) err = E_JACOBIAN;
            double rad = 1.0;
            if (A.axisym) {
                rad = 0.0;
#pragma unroll
                for (int m = 0; m < NN; m++) rad += Ns[m * 16 + p] * Xs[m * 2];
            }
            const double coef = det * ws[p] * (A.axisym ? rad : A.thickness);
            double eps[4] = {0.0, 0.0, 0.0, 0.0};
            double* Gp = G + p * GS;
#pragma unroll
            for (int m = 0; m < NN; m++) {
                double g[2];
#pragma unroll
                for (int i = 0; i < 2; i++) {
                    double v = 0.0;
#pragma unroll
                    for (int j = 0; j < 2; j++) v = fma(dNs[(m * 2 + j) * 16 + p], Ji[j * 2 + i], v);
                    g[i] = v;
                }
                reinterpret_cast<double2*>(Gp)[m] = make_double2(g[0], g[1]);
                if (do_update) {
                    const double* u = Us + m * 2;
                    eps[0] += u[0] * g[0];
                    eps[1] += u[1] * g[1];
                    eps[3] += SQRT2 * ((u[0] * g[1] + u[1] * g[0]) / 2.0);
                }
            }
            if (A.axisym && do_update)  // out-of-plane strain u_r / r (calculate_strain.rs:36-48)
#pragma unroll
                for (int m = 0; m < NN; m++) eps[2] += Us[m * 2] * Ns[m * 16 + p] / rad;
            if (do_update) {
                const int st = ip_update<4>(mc, mc.hh, sig, z, lam, el, eps);
                if (st != OK && err == OK) err = st;
            }
            if (DOF) {  // coef * sigma: xx, yy, xy, hoop (axisymmetric), and the radius
                double* c6 = CS + p * 6;
                c6[0] = coef * sig[0];
                c6[1] = coef * sig[1];
                c6[2] = coef * sig[3] * INV_SQRT2;
                c6[3] = coef * sig[2];
                c6[4] = rad;
            }
            if (dok_c) {
                double a, b, s[4];
                err_t = tangent_coefs<4>(mc, mc.hh, sig, lam, el, a, b, s);
                double* t = TC + p * 4;
                t[0] = coef * 0.5 * a;
                // volumetric coefficient: K - a/3 (= Lame lambda when elastic); plane stress: lambda*
                t[1] = coef * (mc.plane_stress ? mc.ps12 : (mc.kk - a / 3.0));
                t[2] = coef * b;
                const bool plastic = t[2] != 0.0;
                const double s00 = s[0], s11 = s[1], s01 = s[3] * INV_SQRT2, szz = s[2];
                double* Hp = H + p * GS;
                double* Qp = Q + p * NN;
#pragma unroll
                for (int m = 0; m < NN; m++) {
                    const double2 gm = reinterpret_cast<const double2*>(Gp)[m];
                    const double g0 = gm.x, g1 = gm.y;
                    double q = 0.0;  // N/r of node m (axisymmetric)
                    if (A.axisym) {
                        q = Ns[m * 16 + p] / rad;
                        Qp[m] = q;
                    }
                    double h0 = 0.0, h1 = 0.0;  // h = S g (+ q s_zz e_x)
                    if (plastic) {
                        h0 = fma(s00, g0, h0);
                        h0 = fma(s01, g1, h0);
                        h1 = fma(s01, g0, h1);
                        h1 = fma(s11, g1, h1);
                        if (A.axisym) h0 = fma(q, szz, h0);
                    }
                    reinterpret_cast<double2*>(Hp)[m] = make_double2(h0, h1);
                }
            }
        }
        // first failing IP of each cell (lowest p): an update error if any, else a tangent error
        {
            const unsigned bad = __ballot_sync(FULL, err != OK);
            const unsigned bad_t = __ballot_sync(FULL, err_t != OK);
            const unsigned mine = (bad >> (LPC * hh)) & ((1u << LPC) - 1u);
            const unsigned mine_t = (bad_t >> (LPC * hh)) & ((1u << LPC) - 1u);
            const int first = mine ? __ffs(mine) - 1 : 0;
            const int first_t = mine_t ? __ffs(mine_t) - 1 : 0;
            const int code = __shfl_sync(FULL, err, LPC * hh + first);
            const int code_t = __shfl_sync(FULL, err_t, LPC * hh + first_t);
            if (active && hl == 0) {
                if (mine) report(A, do_update ? RANK_UPDATE : RANK_TANGENT, code, cell, first);
                else if (mine_t) report(A, RANK_TANGENT, code_t, cell, first_t);
            }
        }
        if (active && do_update && has_ip) {
#pragma unroll
            for (int c = 0; c < 4; c++) A.sig[(int64_t)c * A.nip + ip0 + hl] = sig[c];
            A.z[ip0 + hl] = z;
            A.lam[ip0 + hl] = lam;
            A.el[ip0 + hl] = (uint8_t)el;
        }
        __syncwarp();

        // ---------------- F_int: lane m of the half owns node m ----------------
        if (DOF && hl < NN) {
            double f[2] = {0.0, 0.0};
            for (int p = 0; p < ng; p++) {
                const double* c6 = CS + p * 6;
                const double* g = G + p * GS + hl * 2;
                f[0] += c6[0] * g[0] + c6[2] * g[1];
                f[1] += c6[2] * g[0] + c6[1] * g[1];
                if (A.axisym) f[0] += c6[3] * Ns[hl * 16 + p] / c6[4];
            }
            if (CSR) {  // kept in the cell's dU slot (free after phase 1) until the scatter
                Us[hl * 2] = f[0];
                Us[hl * 2 + 1] = f[1];
            } else if (active) {
                A.fe[((cell - A.ke_cell0) * NN + hl) * 2] = f[0];
                A.fe[((cell - A.ke_cell0) * NN + hl) * 2 + 1] = f[1];
            }
        }

        if constexpr (CSR) {
            if ((DOF || DOK) && active) {  // the scatter's row data and slot map, copied during phase 2
                if (hl < NN) {
                    const int64_t pt = A.conn[cell * NN + hl];
                    int64_t* nm = NM + 4 * hl;
                    cp_async<8>(nm, A.bptr + pt);
                    cp_async<8>(nm + 1, A.bptr + pt + 1);
                    cp_async<4>(nm + 2, A.crank + cell * NN + hl);
                    cp_async<4>(reinterpret_cast<int32_t*>(nm + 2) + 1, A.cfirst + cell * NN + hl);
                    nm[3] = pt;
                }
                constexpr int CB = NN * NN * 2;
                const char* src = reinterpret_cast<const char*>(A.cslot + cell * (int64_t)(NN * NN));
                char* dst = reinterpret_cast<char*>(CSL);
                if (hl < LPC) {
                    if constexpr (CB % 16 == 0) {
                        for (int k = hl; k < CB / 16; k += LPC) cp_async<16>(dst + 16 * k, src + 16 * k);
                    } else if constexpr (CB % 8 == 0) {
                        for (int k = hl; k < CB / 8; k += LPC) cp_async<8>(dst + 8 * k, src + 8 * k);
                    } else {  // a map whose cell offset is not 4-byte aligned (Tri3, Qua9): plain loads
                        for (int k = hl; k < NN * NN; k += LPC) CSL[k] = A.cslot[cell * (int64_t)(NN * NN) + k];
                    }
                }
            }
        }
        // ---------------- phase 2: lane owns a tile of node-pair blocks ----------------
        double acc[T][T][2][2];
        if (DOK) {
            const int a0 = ti * T, b0 = tj * T;
#pragma unroll
            for (int r = 0; r < T; r++)
#pragma unroll
                for (int c = 0; c < T; c++)
#pragma unroll
                    for (int i = 0; i < 2; i++)
#pragma unroll
                        for (int j = 0; j < 2; j++) acc[r][c][i][j] = 0.0;
            if (dok_c && ti >= 0 && !A.axisym) {
                // two passes, as in element_kernel: X_ab = sum_p alpha_p g_a g_b^T over every point,
                // K_ab = X_ab^T + tr(X_ab) 1 + c X_ab, then kappa_p g_a g_b^T + beta_p h_a h_b^T at
                // the plastic points (c = gamma/alpha of the elastic tangent, kappa = gamma - c alpha)
                const double cvol = (mc.plane_stress ? mc.ps12 : mc.kk - 2.0 * mc.gg / 3.0) / mc.gg;
                for (int p = 0; p < ng; p++) {
                    const double al = TC[p * 4];
                    const double2* Gp = reinterpret_cast<const double2*>(G + p * GS);
                    double ar[T][2];
#pragma unroll
                    for (int r = 0; r < T; r++) {
                        const double2 ga2 = Gp[min(a0 + r, NN - 1)];
                        ar[r][0] = al * ga2.x;
                        ar[r][1] = al * ga2.y;
                    }
#pragma unroll
                    for (int c = 0; c < T; c++) {
                        const double2 gb2 = Gp[min(b0 + c, NN - 1)];
                        const double gb[2] = {gb2.x, gb2.y};
#pragma unroll
                        for (int r = 0; r < T; r++)
#pragma unroll
                            for (int i = 0; i < 2; i++)
#pragma unroll
                                for (int j = 0; j < 2; j++) acc[r][c][i][j] = fma(ar[r][i], gb[j], acc[r][c][i][j]);
                    }
                }
#pragma unroll
                for (int r = 0; r < T; r++)
#pragma unroll
                    for (int c = 0; c < T; c++) {
                        const double x00 = acc[r][c][0][0], x01 = acc[r][c][0][1];
                        const double x10 = acc[r][c][1][0], x11 = acc[r][c][1][1];
                        const double tr = x00 + x11;
                        acc[r][c][0][0] = fma(cvol, x00, x00) + tr;
                        acc[r][c][0][1] = fma(cvol, x01, x10);
                        acc[r][c][1][0] = fma(cvol, x10, x01);
                        acc[r][c][1][1] = fma(cvol, x11, x11) + tr;
                    }
                for (int p = 0; p < ng; p++) {
                    const double2 t01 = reinterpret_cast<const double2*>(TC)[2 * p];
                    const double be = TC[p * 4 + 2];
                    if (be == 0.0) continue;  // elastic point
                    const double kap = t01.y - cvol * t01.x;
                    const double2* Gp = reinterpret_cast<const double2*>(G + p * GS);
                    const double2* Hp = reinterpret_cast<const double2*>(H + p * GS);
                    double kr[T][2], hr[T][2];
#pragma unroll
                    for (int r = 0; r < T; r++) {
                        const int a = min(a0 + r, NN - 1);
                        const double2 ga2 = Gp[a], ha2 = Hp[a];
                        kr[r][0] = kap * ga2.x;
                        kr[r][1] = kap * ga2.y;
                        hr[r][0] = be * ha2.x;
                        hr[r][1] = be * ha2.y;
                    }
#pragma unroll
                    for (int c = 0; c < T; c++) {
                        const int b = min(b0 + c, NN - 1);
                        const double2 gb2 = Gp[b], hb2 = Hp[b];
                        const double gb[2] = {gb2.x, gb2.y};
                        const double hb[2] = {hb2.x, hb2.y};
#pragma unroll
                        for (int r = 0; r < T; r++)
#pragma unroll
                            for (int i = 0; i < 2; i++)
#pragma unroll
                                for (int j = 0; j < 2; j++) {
                                    acc[r][c][i][j] = fma(kr[r][i], gb[j], acc[r][c][i][j]);
                                    acc[r][c][i][j] = fma(hr[r][i], hb[j], acc[r][c][i][j]);
                                }
                    }
                }
            } else if (dok_c && ti >= 0) {  // axisymmetric: the hoop terms take the one-pass form
                for (int p = 0; p < ng; p++) {
                    const double2 t01 = reinterpret_cast<const double2*>(TC)[2 * p];
                    const double al = t01.x, ga = t01.y, be = TC[p * 4 + 2];
                    const bool plastic = be != 0.0;
                    const double* Gp = G + p * GS;
                    const double* Hp = H + p * GS;
                    const double* Qp = Q + p * NN;
                    double Ar[T][2], Cr[T][2], Hr[T][2], Qr[T];
#pragma unroll
                    for (int r = 0; r < T; r++) {
                        const int a = min(a0 + r, NN - 1);
                        const double2 ga2 = reinterpret_cast<const double2*>(Gp)[a];
                        const double2 ha2 = reinterpret_cast<const double2*>(Hp)[a];
                        const double g0 = ga2.x, g1 = ga2.y;
                        const double q = A.axisym ? Qp[a] : 0.0;
                        Ar[r][0] = al * g0;
                        Ar[r][1] = al * g1;
                        Cr[r][0] = ga * (A.axisym ? g0 + q : g0);
                        Cr[r][1] = ga * g1;
                        Hr[r][0] = be * ha2.x;
                        Hr[r][1] = be * ha2.y;
                        Qr[r] = 2.0 * al * q;
                    }
#pragma unroll
                    for (int c = 0; c < T; c++) {
                        const int b = min(b0 + c, NN - 1);
                        const double2 gb2 = reinterpret_cast<const double2*>(Gp)[b];
                        const double2 hb2 = reinterpret_cast<const double2*>(Hp)[b];
                        const double gb[2] = {gb2.x, gb2.y};
                        const double hb[2] = {hb2.x, hb2.y};
                        const double qb = A.axisym ? Qp[b] : 0.0;
                        const double gc[2] = {A.axisym ? gb[0] + qb : gb[0], gb[1]};
                        double dot[T];
#pragma unroll
                        for (int r = 0; r < T; r++) {
                            dot[r] = 0.0;
#pragma unroll
                            for (int k = 0; k < 2; k++) dot[r] = fma(Ar[r][k], gb[k], dot[r]);
                        }
#pragma unroll
                        for (int r = 0; r < T; r++)
#pragma unroll
                            for (int i = 0; i < 2; i++)
#pragma unroll
                                for (int j = 0; j < 2; j++) acc[r][c][i][j] = fma(Ar[r][j], gb[i], acc[r][c][i][j]);
#pragma unroll
                        for (int r = 0; r < T; r++)
#pragma unroll
                            for (int i = 0; i < 2; i++)
#pragma unroll
                                for (int j = 0; j < 2; j++) acc[r][c][i][j] = fma(Cr[r][i], gc[j], acc[r][c][i][j]);
                        if (plastic) {
#pragma unroll
                            for (int r = 0; r < T; r++)
#pragma unroll
                                for (int i = 0; i < 2; i++)
#pragma unroll
                                    for (int j = 0; j < 2; j++) acc[r][c][i][j] = fma(Hr[r][i], hb[j], acc[r][c][i][j]);
                        }
#pragma unroll
                        for (int r = 0; r < T; r++)
#pragma unroll
                            for (int i = 0; i < 2; i++) acc[r][c][i][i] += dot[r];
                        if (A.axisym)  // hoop row: a (N_a/r)(N_b/r) on the radial-radial entry
#pragma unroll
                            for (int r = 0; r < T; r++) acc[r][c][0][0] = fma(Qr[r], qb, acc[r][c][0][0]);
                    }
                }
            }
            if constexpr (!CSR) {  // dense output
            __syncwarp();  // both halves are done reading the cell areas that the staging overwrites
            // stage K_e row-major in the cell area (blocks (a, b) and their mirrors (b, a)), then
            // copy it out with 16-byte stores, LPC*16 contiguous bytes per cell and store
            double* stage = Xs;
            constexpr int NU = NN * (NN + 1) / 2;  // upper layout: blocks (a <= b), 2x2 each
            const bool up = A.ke_upper != 0;
            if (ti >= 0) {
#pragma unroll
                for (int r = 0; r < T; r++)
#pragma unroll
                    for (int c = 0; c < T; c++) {
                        const int a = a0 + r, b = b0 + c;
                        if (a < NN && b < NN && a <= b) {
                            if (up) {
#pragma unroll
                                for (int i = 0; i < 2; i++)
#pragma unroll
                                    for (int j = 0; j < 2; j++) stage[upper_entry<NN, 2>(a, b, i, j)] = acc[r][c][i][j];
                            } else {
#pragma unroll
                                for (int i = 0; i < 2; i++)
#pragma unroll
                                    for (int j = 0; j < 2; j++) {
                                        stage[(a * 2 + i) * NE + b * 2 + j] = acc[r][c][i][j];
                                        if (a != b) stage[(b * 2 + j) * NE + a * 2 + i] = acc[r][c][i][j];
                                    }
                            }
                        }
                    }
            }
            __syncwarp();
            if (active && hl < LPC) {
                const int nd2 = up ? 2 * NU : NE * NE / 2;  // double2 per cell
                double2* dst = reinterpret_cast<double2*>(A.ke + (cell - A.ke_cell0) * (int64_t)(2 * nd2));
                const double2* s2 = reinterpret_cast<const double2*>(stage);
                for (int t = hl; t < nd2; t += LPC) dst[t] = s2[t];
            }
            }  // dense output
        }
        // ---------------- direct assembly: ordered scatter into the CSR values and R ----------------
        // As in element_kernel, with the CPW cells of the warp in one round structure: each slot stages
        // its cell's upper blocks after its dU slot (which holds F_int), node lane (slot h, node m)
        // takes row conn[m] of cell h once the row's ticket equals that cell's rank, and for every
        // ready row the whole warp writes the row's values (nodes in ascending id, so consecutive
        // lanes write consecutive CSR positions).  A row shared by two cells of the warp is added by
        // the one earlier in the processing order first (its rank is lower).  Slots without a cell
        // add nothing.
        if constexpr (CSR) {
            if (DOF || DOK) {
                double* KS = Us + NE;  // this slot's upper blocks (2x2 each, upper_entry layout)
                {
                    const int a0 = max(ti, 0) * T, b0 = max(tj, 0) * T;
                    if (dok_c && ti >= 0) {
#pragma unroll
                        for (int r = 0; r < T; r++)
#pragma unroll
                            for (int c = 0; c < T; c++) {
                                const int a = a0 + r, b = b0 + c;
                                if (a < NN && b < NN && a <= b) {
#pragma unroll
                                    for (int i = 0; i < 2; i++)
#pragma unroll
                                        for (int j = 0; j < 2; j++) KS[upper_entry<NN, 2>(a, b, i, j)] = acc[r][c][i][j];
                                }
                            }
                    }
                }
                cp_async_wait_all();
                __syncwarp();  // the staged blocks and every lane's copies are visible
                // release the rows the slot's previous cell left pending before anything can wait here
                if (hl < NN && PEND[2 * hl] >= 0) {
                    ticket_store(A.ticket + PEND[2 * hl], (int)PEND[2 * hl + 1]);
                    PEND[2 * hl] = -1;
                }
                int64_t rowA = INT64_MAX, pos_m = 0;
                int rs_m = 0, rank_m = 0;
                bool last_m = false, todo = false;
                if (active && hl < NN) {
                    const int64_t* nm = NM + 4 * hl;
                    rowA = nm[3];
                    const int64_t r0 = nm[0], r1 = nm[1];
                    pos_m = 4 * r0;
                    rs_m = 2 * (int)(r1 - r0);
                    const int32_t cr = reinterpret_cast<const int32_t*>(nm + 2)[0];
                    rank_m = cr & CRANK_MASK;
                    last_m = (cr & CRANK_LAST) != 0;
                    todo = true;
                }
                {  // each slot's local nodes in ascending node id
                    const int sb = LPC * hh;
                    int rk = 0;
#pragma unroll
                    for (int q = 0; q < NN; q++) rk += __shfl_sync(FULL, rowA, sb + q) < rowA;
                    if (active && hl < NN) CSORT[rk] = (uint8_t)hl;
                }
                __syncwarp();
                const double* ks_base = smem2 + table2_doubles(NN) + (int64_t)(CPW * wid) * cd + 2 * NE;
                const unsigned dokmask = __ballot_sync(FULL, dok_c);  // the slots whose K rows are written
                const int64_t* nm_base = reinterpret_cast<const int64_t*>(smem2 + table2_doubles(NN) + CPW * WPB2 * cd +
                                                                         (CPW * wid) * meta_doubles(NN));
                int spins = 0;
                while (true) {
                    const unsigned todo_mask = __ballot_sync(FULL, todo);
                    if (!todo_mask) break;
                    bool ready = todo && ticket_load(A.ticket + rowA) == rank_m;
                    unsigned rmask = __ballot_sync(FULL, ready);
                    if (!rmask) {
                        ++spins;
                        const bool give_up = __shfl_sync(FULL, spins >= ORDER_WAIT_LIMIT || ((spins & 63) == 0 && order_aborted(A.errkey)), 0);
                        if (!give_up) {
                            __nanosleep(order_backoff(spins));
                            continue;
                        }
                        if (lane == 0) report(A, RANK_ORDER, E_ORDER, cell, 0);
                        ready = todo;
                        rmask = todo_mask;
                    }
                    __syncwarp();  // the node lanes' acquires order every lane's writes after the earlier cells'
                    if (DOF && ready) {
#pragma unroll
                        for (int i = 0; i < 2; i++) {
                            double* q = A.ff + rowA * 2 + i;
                            if (rank_m == 0) *q = 0.0 + Us[hl * 2 + i];
                            else red_add(q, Us[hl * 2 + i]);
                        }
                    }
                    if (DOK) {
                        for (unsigned rows = rmask & dokmask; rows; rows &= rows - 1) {  // the ready rows
                            const int bit = __ffs(rows) - 1;
                            const int h = bit / LPC, a = bit - h * LPC;  // slot and local node of the row
                            const int64_t pa = __shfl_sync(FULL, pos_m, bit);
                            const int rsa = __shfl_sync(FULL, rs_m, bit);
                            const double* ks = ks_base + (int64_t)h * cd;
                            const int64_t* nm = nm_base + (int64_t)h * (meta_doubles(NN));
                            const int16_t* csl = reinterpret_cast<const int16_t*>(nm + 6 * NN);
                            const uint8_t* cso = reinterpret_cast<const uint8_t*>(csl) + 16 * ((NN * NN + 7) / 8);
                            const uint32_t fa = reinterpret_cast<const uint32_t*>(nm + 4 * a + 2)[1];
                            for (int e = lane; e < 2 * NN * 2; e += 32) {
                                const int i = e / (NN * 2), k = (e - i * NN * 2) / 2, j = e - i * NN * 2 - k * 2;
                                const int b = cso[k];
                                const double v = (a <= b) ? ks[upper_entry<NN, 2>(a, b, i, j)] : ks[upper_entry<NN, 2>(b, a, j, i)];
                                double* q = A.csr + pa + (int64_t)i * rsa + 2 * (int64_t)csl[a * NN + b] + j;
                                if ((fa >> b) & 1u) *q = 0.0 + v;
                                else red_add(q, v);
                            }
                        }
                    }
                    __syncwarp();  // every lane's writes precede the node lanes' (cumulative) release stores
                    // the last round's rows are released at the slot's next scatter (or the exit)
                    const bool final = rmask == todo_mask;
                    if (ready) {
                        if (final) {
                            PEND[2 * hl] = rowA;
                            PEND[2 * hl + 1] = last_m ? 0 : rank_m + 1;
                        } else {
                            ticket_store(A.ticket + rowA, last_m ? 0 : rank_m + 1);
                        }
                    }
                    todo = todo && !ready;
                }
            }
        }
    }  // pairs
    if constexpr (CSR) {  // the last cells' pending releases
        if (hl < NN && PEND[2 * hl] >= 0) ticket_store(A.ticket + PEND[2 * hl], (int)PEND[2 * hl + 1]);
    }
}

// One warp per G = 32/NN consecutive block rows of K (a work-queue range may cut the run); group g
// of NN lanes owns row A_g.  Lane b of the group loads, for each incidence k of A_g (cell c, local
// index a), the ND x ND block (a, b) of c's element matrix -- kept as its upper blocks, block row by
// block row, so lane b reads block (a, b) when a <= b (the lanes b >= a read adjacent segments of
// the same scalar rows) and the transpose of block (b, a) otherwise -- and adds it at column
// slot[k*NN + b] of the row's buffer in shared memory.  Up
// to NB incidences are loaded before they are added; the adds go in ascending incidence (= cell)
// order with a group barrier between incidences, so every entry of K is the fixed-order sum over
// its cells: bit-identical on every run.  The G buffers lie back to back in CSR order, so when the
// rows are consecutive the warp writes them out as one contiguous run.  Rows of problems whose mode
// is 0 are skipped (per-problem batches).
template <int ND, int NN> struct GatherShape {
    static constexpr int G = NN >= 32 ? 1 : 32 / NN;  // rows per warp
    static constexpr int NB = 4;                      // incidences loaded before they are added
};

// TRI: the CSR values hold one triangle of K (sym = PMS_SYM_LOWER: columns <= row, PMS_SYM_UPPER:
// columns >= row; src/base/assembly.rs:92-122): the lanes skip the blocks that fall outside it, and
// row (A, i) starts at tbase[A] plus the lengths of rows (A, 0..i-1); kdiag[A] = A's own position
// in its block row.
template <int ND, int NN, bool TRI>
__global__ void __launch_bounds__(256, ND == 2 ? 4 : 1) kk_gather_kernel(int64_t npoint, int nbmax, const int64_t* __restrict__ bptr,
                                                        const int64_t* __restrict__ inc_ptr,
                                                        const int32_t* __restrict__ inc,
                                                        const int16_t* __restrict__ slot,
                                                        const double* __restrict__ ke, double* __restrict__ csr,
                                                        const int32_t* __restrict__ node_prob,
                                                        const uint8_t* __restrict__ pmode, int nq,
                                                        const int64_t* __restrict__ q_off,
                                                        const int64_t* __restrict__ q_first, int64_t node0,
                                                        int sym, const int32_t* __restrict__ kdiag,
                                                        const int64_t* __restrict__ tbase) {
    constexpr int BB = ND * ND, NU = NN * (NN + 1) / 2;
    constexpr int G = GatherShape<ND, NN>::G, NB = GatherShape<ND, NN>::NB;
    extern __shared__ double rowbuf[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    double* buf = rowbuf + (int64_t)wid * G * nbmax * BB;
    const int g = lane / NN, b = lane - (lane / NN) * NN;
    const bool lane_on = g < G;
    const unsigned gmask = lane_on ? (((NN >= 32) ? 0xffffffffu : ((1u << NN) - 1u)) << (g * NN)) : (1u << lane);
    const int64_t ngroup = (npoint + G - 1) / G;
    const int64_t nwarp = (int64_t)gridDim.x * wpb;
    for (int64_t w = (int64_t)blockIdx.x * wpb + wid; w < ngroup; w += nwarp) {
        const int64_t Ai = w * G + g;
        bool on = lane_on && Ai < npoint;
        int64_t A = 0;
        if (on) {
            A = nq ? queue_item(Ai, nq, q_off, q_first) : node0 + Ai;
            if (pmode && pmode[node_prob[A]] == 0) on = false;
        }
        int64_t ba = 0;
        int nba = 0, dp = 0;
        if (on) {
            ba = bptr[A];
            nba = (int)(bptr[A + 1] - ba);
            if constexpr (TRI) dp = kdiag[A];
        }
        // buffer offsets of the group rows (exclusive scan over the groups) and the run test
        int off = 0, total = 0;
#pragma unroll
        for (int q = 0; q < G; q++) {
            const int nq_ = __shfl_sync(FULL, nba, q * NN);
            if (q < g) off += nq_;
            total += nq_;
        }
        const int64_t A0 = __shfl_sync(FULL, A, 0);
        const bool on0 = __shfl_sync(FULL, on, 0);
        const bool fits = !lane_on || Ai >= npoint || (on && A == A0 + g);
        const bool run = !TRI && __all_sync(FULL, fits) && on0;
        for (int t = lane; t < total * BB; t += 32) buf[t] = 0.0;
        __syncwarp();
        if (on) {
            double* rb = buf + (int64_t)off * BB;
            const int nrow = ND * nba;
            const int64_t k0 = inc_ptr[A], k1 = inc_ptr[A + 1];
            for (int64_t kb = k0; kb < k1; kb += NB) {
                double v[NB][BB];
                int pos[NB];
#pragma unroll
                for (int r = 0; r < NB; r++) {
                    const int64_t k = kb + r;
                    pos[r] = -1;
                    if (k < k1) {
                        const int32_t code = __ldg(inc + k);
                        const int64_t cell = code / NN;
                        const int a = code - (int)cell * NN;
                        pos[r] = __ldg(slot + k * NN + b);
                        if constexpr (TRI) {
                            if (sym == PMS_SYM_LOWER ? pos[r] > dp : pos[r] < dp) {
                                pos[r] = -1;  // outside the stored triangle: neither loaded nor added
#pragma unroll
                                for (int i = 0; i < BB; i++) v[r][i] = 0.0;
                                continue;
                            }
                        }
                        // block (a, b) of the upper layout: stored as (a, b) when a <= b, else as (b, a);
                        // the lanes b >= a read adjacent segments of the same scalar rows
                        const bool upper = a <= b;
                        const int lo = upper ? a : b, hi = upper ? b : a;
                        const double* src = ke + cell * (int64_t)(NU * BB) + upper_entry<NN, ND>(lo, hi, 0, 0);
                        const int rs = (NN - lo) * ND;  // scalar-row stride of block row lo
#pragma unroll
                        for (int i = 0; i < ND; i++)
#pragma unroll
                            for (int j = 0; j < ND; j++) v[r][i * ND + j] = __ldg(src + (upper ? i * rs + j : j * rs + i));
                    } else {
#pragma unroll
                        for (int i = 0; i < BB; i++) v[r][i] = 0.0;
                    }
                }
#pragma unroll
                for (int r = 0; r < NB; r++) {
                    __syncwarp(gmask);  // the group's previous incidence is added
                    if (pos[r] >= 0) {
#pragma unroll
                        for (int i = 0; i < ND; i++)
#pragma unroll
                            for (int j = 0; j < ND; j++) rb[i * nrow + pos[r] * ND + j] += v[r][i * ND + j];
                    }
                }
            }
        }
        __syncwarp();
        if (run) {
            double* dst = csr + (int64_t)BB * __shfl_sync(FULL, ba, 0);
            for (int t = lane; t < total * BB; t += 32) dst[t] = buf[t];
        } else if constexpr (TRI) {
            // buffer entry (i, c = p*ND + j) of a row group is K(A*ND + i, B_p*ND + j).  The group's
            // stored entries are contiguous from tbase[A]: row i holds, lower, c = 0 .. ND*dq + i
            // (from i*ND*dq + i(i+1)/2 on), upper, c = dq*ND + i .. ND*nq - 1 (from
            // i*ND*(nq - dq) - i(i-1)/2 on); each lane takes destinations and finds their row
            const bool lower = sym == PMS_SYM_LOWER;
            const int64_t tb = on ? tbase[A] : 0;
            int oq = 0;
#pragma unroll 1
            for (int q = 0; q < G; q++) {
                const int nq_ = __shfl_sync(FULL, nba, q * NN);
                const int dq = __shfl_sync(FULL, dp, q * NN);
                double* dst = csr + __shfl_sync(FULL, tb, q * NN);
                const double* src = buf + (int64_t)oq * BB;
                const int nrow = ND * nq_, w = lower ? ND * dq : ND * (nq_ - dq);
                const int cnt = nq_ ? (lower ? BB * dq : BB * (nq_ - dq - 1)) + ND * (ND + 1) / 2 : 0;
                for (int u = lane; u < cnt; u += 32) {
                    int i = 0, s0 = 0;
#pragma unroll
                    for (int ii = 1; ii < ND; ii++) {
                        const int s = lower ? ii * w + ii * (ii + 1) / 2 : ii * w - ii * (ii - 1) / 2;
                        if (u >= s) i = ii, s0 = s;
                    }
                    dst[u] = src[i * nrow + (u - s0) + (lower ? 0 : dq * ND + i)];
                }
                oq += nq_;
            }
        } else {
            int oq = 0;
#pragma unroll 1
            for (int q = 0; q < G; q++) {
                const int nq_ = __shfl_sync(FULL, nba, q * NN);
                const int64_t bq = __shfl_sync(FULL, ba, q * NN);
                double* dst = csr + (int64_t)BB * bq;  // rows that are absent or inactive have nq_ = 0
                const double* src = buf + (int64_t)oq * BB;
                for (int t = lane; t < nq_ * BB; t += 32) dst[t] = src[t];
                oq += nq_;
            }
        }
        __syncwarp();
    }
}

// One thread per point: R[A*nd + i] = sum over its incidences (ascending cell) of f_e.
template <int ND>
__global__ void __launch_bounds__(256) f_gather_kernel(int64_t npoint, const int64_t* __restrict__ inc_ptr,
                                                       const int32_t* __restrict__ inc,
                                                       const double* __restrict__ fe, double* __restrict__ ff,
                                                       int nq = 0, const int64_t* __restrict__ q_off = nullptr,
                                                       const int64_t* __restrict__ q_first = nullptr) {
    for (int64_t Ai = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; Ai < npoint;
         Ai += (int64_t)gridDim.x * blockDim.x) {
        const int64_t A = nq ? queue_item(Ai, nq, q_off, q_first) : Ai;
        double s[ND];
#pragma unroll
        for (int i = 0; i < ND; i++) s[i] = 0.0;
        for (int64_t k = inc_ptr[A]; k < inc_ptr[A + 1]; k++) {
            const double* v = fe + (int64_t)inc[k] * ND;
#pragma unroll
            for (int i = 0; i < ND; i++) s[i] += v[i];
        }
#pragma unroll
        for (int i = 0; i < ND; i++) ff[A * ND + i] = s[i];
    }
}

__global__ void init_state_kernel(int64_t nip, int nc, const MatConst* mats, const int32_t* cmat, int ng,
                                  double* sig, double* z, double* lam, uint8_t* el) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nip; i += (int64_t)gridDim.x * blockDim.x) {
        for (int c = 0; c < nc; c++) sig[(int64_t)c * nip + i] = 0.0;
        const MatConst m = mats[cmat ? cmat[i / ng] : 0];
        z[i] = (m.model == 1) ? m.z_ini : 0.0;
        lam[i] = 0.0;
        el[i] = 1;
    }
}

__global__ void zero_lambda_kernel(int64_t nip, double* lam) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nip; i += (int64_t)gridDim.x * blockDim.x)
        lam[i] = 0.0;
}

}  // namespace

// ------------------------------------------------------------------------------- handle
struct pms_elements {
    int nd = 0, kind = 0, nn = 0, ng = 0, nc = 0;
    int gather_wpb = 8, gather_smem = 0;  // rows (warps) per block and shared memory of kk_gather
    int64_t npoint = 0, ncell = 0, ndof = 0, nip = 0, nnz = 0;
    double thickness = 1.0;
    int axisym = 0;
    std::vector<MatConst> mats;
    Pattern pat;
    std::vector<double> tab;  // dN table + weights
    // device buffers
    double* d_coords = nullptr;
    int32_t* d_conn = nullptr;
    int32_t* d_cmat = nullptr;
    MatConst* d_mats = nullptr;
    double* d_tab = nullptr;
    double *d_sig = nullptr, *d_z = nullptr, *d_lam = nullptr;
    uint8_t* d_el = nullptr;
    double *d_sig_b = nullptr, *d_z_b = nullptr, *d_lam_b = nullptr;
    uint8_t* d_el_b = nullptr;
    double* d_fe = nullptr;  // dense F_e / K_e of every cell (gather assembly only; allocated on first use)
    double* d_ke = nullptr;
    double* d_fe1 = nullptr;  // dense F_e / K_e of one cell (per-cell calls)
    double* d_ke1 = nullptr;
    int16_t* d_cslot = nullptr;    // direct assembly: per-cell slot map
    int32_t* d_crank = nullptr;    // direct assembly: per-cell incidence ranks
    uint32_t* d_cfirst = nullptr;  // direct assembly: per-cell first-contribution bits
    int32_t* d_order = nullptr;    // direct assembly: processing order of the cells
    int32_t* d_ticket = nullptr;   // direct assembly: per-node tickets (zero between launches)
    unsigned long long* d_next = nullptr;  // direct assembly: in-order work counter
    int assembly = PMS_ASSEMBLY_GATHER;  // measured faster on B200 for every kind benchmarked
    int sym = PMS_SYM_FULL;              // storage of the public CSR values (pms_elements_set_symmetry)
    std::vector<int64_t> tbase;          // triangle layouts: first value of each node's rows [npoint + 1]
    int64_t* d_tbase = nullptr;
    int64_t* d_inc_ptr = nullptr;
    int32_t* d_inc = nullptr;
    int64_t* d_bptr = nullptr;
    int32_t* d_bcol = nullptr;
    int32_t* d_kdiag = nullptr;
    int16_t* d_slot = nullptr;
    double *d_ddu = nullptr, *d_ff = nullptr, *d_csr = nullptr;  // staging for host-memory calls
    int64_t* d_indptr = nullptr;  // device CSR pattern (built on first request)
    int32_t* d_indices = nullptr;
    int32_t* d_status = nullptr;
    int64_t device_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    std::string last_error;
    int64_t err_cell = -1;
    int32_t err_ip = -1;
    int64_t launches = 0;
    int smem_bytes = 0;
    std::vector<void*> allocs;
    // host-memory calls: the CSR values leave in row slabs on copy_stream while later slabs gather
    static constexpr int NSLAB = 8;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t slab_ev[NSLAB + 1] = {};
    // optional CUDA-event timing of the three kernels of a batched call
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_pool, ev_pending[3];

    template <typename T>
    bool alloc(T** p, size_t count) {
        *p = nullptr;
        if (count == 0) count = 1;
        std::lock_guard<std::mutex> lock(device_mutex());
        if (cudaMalloc((void**)p, count * sizeof(T)) != cudaSuccess) return false;
        allocs.push_back((void*)*p);
        device_bytes += (int64_t)(count * sizeof(T));
        return true;
    }
    template <typename T>
    bool upload(T** p, const T* src, size_t count) {
        if (!alloc(p, count)) return false;
        if (count && cudaMemcpy(*p, src, count * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return false;
        return true;
    }
    std::pair<cudaEvent_t, cudaEvent_t> event_pair() {
        if (!ev_pool.empty()) {
            auto e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        std::pair<cudaEvent_t, cudaEvent_t> e;
        cudaEventCreate(&e.first);
        cudaEventCreate(&e.second);
        return e;
    }
    ~pms_elements() {
        if (own_stream) cudaStreamSynchronize(own_stream);
        std::lock_guard<std::mutex> lock(device_mutex());
        for (auto& v : ev_pending)
            for (auto& e : v) ev_pool.push_back(e);
        for (auto& e : ev_pool) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        if (copy_stream) {
            cudaStreamSynchronize(copy_stream);
            for (auto& e : slab_ev)
                if (e) cudaEventDestroy(e);
            cudaStreamDestroy(copy_stream);
        }
        for (void* p : allocs) cudaFree(p);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace {

int fail(pms_elements* h, int code, const char* msg) {
    if (h) h->last_error = msg;
    return code;
}

int cuda_check(pms_elements* h) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, PMS_ERR_CUDA, cudaGetErrorString(e));
    return PMS_OK;
}

int grid_1d(int64_t n) {
    int64_t b = (n + 255) / 256;
    if (b > 148 * 16) b = 148 * 16;
    return (int)std::max<int64_t>(b, 1);
}

// Lets a kernel take up to the device's opt-in shared memory per block (each launch still asks for
// its own size, from which the residency is computed).
void allow_dynamic_smem(const void* kern) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
}

// Blocks of a kernel that the GPU holds at once (one wave of the persistent element kernel).
int64_t resident_blocks(const void* kern, int smem, int threads = WPB * 32) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    return (int64_t)std::max(sms, 1) * per_sm;
}

// 2D cells with at most 16 integration points: LPC lanes per cell, 32/LPC cells per warp
template <int NN, int LPC, int UPD, bool DOF, bool DOK, bool CSR>
void launch_elem2d_lpc(const ElemArgs& a, cudaStream_t st, bool persistent) {
    constexpr int CPW = 32 / LPC;
    auto kern = element2d_kernel<NN, LPC, UPD, DOF, DOK, CSR>;
    const int smem = smem2_bytes(NN, a.ngauss, CPW, CSR);
    allow_dynamic_smem((const void*)kern);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    int64_t blocks = ((a.ncell + CPW - 1) / CPW + WPB2 - 1) / WPB2;
    if (persistent || CSR) blocks = std::min<int64_t>(blocks, resident_blocks((const void*)kern, smem, WPB2 * 32));
    if (CSR) cudaMemsetAsync(a.next, 0, sizeof(unsigned long long), st);
    kern<<<(unsigned)std::max<int64_t>(blocks, 1), WPB2 * 32, smem, st>>>(a);
}

template <int NN, int UPD, bool DOF, bool DOK, bool CSR>
void launch_elem2d_t(const ElemArgs& a, cudaStream_t st, bool persistent) {
    if constexpr (packed_layout<NN>()) {
        if (a.ngauss <= lanes_packed<NN>()) {
            launch_elem2d_lpc<NN, lanes_packed<NN>(), UPD, DOF, DOK, CSR>(a, st, persistent);
            return;
        }
    }
    launch_elem2d_lpc<NN, 16, UPD, DOF, DOK, CSR>(a, st, persistent);
}

template <int ND, int NN, int UPD, bool DOF, bool DOK, bool CSR>
void launch_elem_t(pms_elements* h, const ElemArgs& a) {
    if constexpr (ND == 2 && fits_2d<NN>()) {
        if (a.ngauss <= NG2_MAX) {
            launch_elem2d_t<NN, UPD, DOF, DOK, CSR>(a, h->stream, true);
            return;
        }
    }
    auto kern = element_kernel<ND, NN, UPD, DOF, DOK, CSR>;
    allow_dynamic_smem((const void*)kern);
    int64_t blocks = (a.ncell + cells_per_block(NN) - 1) / cells_per_block(NN);
    blocks = std::min<int64_t>(blocks, resident_blocks((const void*)kern, h->smem_bytes));
    if (CSR) cudaMemsetAsync(a.next, 0, sizeof(unsigned long long), h->stream);
    kern<<<(unsigned)blocks, WPB * 32, h->smem_bytes, h->stream>>>(a);
}

// upd: UPD_NONE / UPD_CURRENT / UPD_BACKUP; csr: direct assembly into a.csr / a.ff (else dense
// fe / ke outputs).  Update-only launches (no output) have no assembly.
template <int ND, int NN>
void launch_elem_nn(pms_elements* h, const ElemArgs& a, int upd, bool dof, bool dok, bool csr) {
    if (!dof && !dok) {
        if (upd == UPD_CURRENT) launch_elem_t<ND, NN, UPD_CURRENT, false, false, false>(h, a);
        else launch_elem_t<ND, NN, UPD_BACKUP, false, false, false>(h, a);
        return;
    }
    if (upd == UPD_NONE) {
        if (csr) {
            if (dof && dok) launch_elem_t<ND, NN, UPD_NONE, true, true, true>(h, a);
            else if (dof) launch_elem_t<ND, NN, UPD_NONE, true, false, true>(h, a);
            else launch_elem_t<ND, NN, UPD_NONE, false, true, true>(h, a);
        } else {
            if (dof && dok) launch_elem_t<ND, NN, UPD_NONE, true, true, false>(h, a);
            else if (dof) launch_elem_t<ND, NN, UPD_NONE, true, false, false>(h, a);
            else launch_elem_t<ND, NN, UPD_NONE, false, true, false>(h, a);
        }
    } else {
        // update from the backup, then the requested outputs (the direct assembly writes exactly
        // those; the dense outputs always go to the handle's own buffers).  Updates of the current
        // state with outputs are not used by any call.
        if (csr) {
            if (dof && dok) launch_elem_t<ND, NN, UPD_BACKUP, true, true, true>(h, a);
            else if (dof) launch_elem_t<ND, NN, UPD_BACKUP, true, false, true>(h, a);
            else launch_elem_t<ND, NN, UPD_BACKUP, false, true, true>(h, a);
        } else {
            launch_elem_t<ND, NN, UPD_BACKUP, true, true, false>(h, a);
        }
    }
}

void launch_elem(pms_elements* h, const ElemArgs& a, int upd, bool dof, bool dok, bool csr) {
    if (upd == UPD_MODE) {  // batched solver: always the direct assembly
        switch (h->kind) {
        case PMS_TRI3: launch_elem_t<2, 3, UPD_MODE, true, true, true>(h, a); break;
        case PMS_TRI6: launch_elem_t<2, 6, UPD_MODE, true, true, true>(h, a); break;
        case PMS_QUA4: launch_elem_t<2, 4, UPD_MODE, true, true, true>(h, a); break;
        case PMS_QUA8: launch_elem_t<2, 8, UPD_MODE, true, true, true>(h, a); break;
        case PMS_QUA9: launch_elem_t<2, 9, UPD_MODE, true, true, true>(h, a); break;
        case PMS_TET4: launch_elem_t<3, 4, UPD_MODE, true, true, true>(h, a); break;
        case PMS_TET10: launch_elem_t<3, 10, UPD_MODE, true, true, true>(h, a); break;
        case PMS_HEX8: launch_elem_t<3, 8, UPD_MODE, true, true, true>(h, a); break;
        case PMS_HEX20: launch_elem_t<3, 20, UPD_MODE, true, true, true>(h, a); break;
        case PMS_TRI10: launch_elem_t<2, 10, UPD_MODE, true, true, true>(h, a); break;
        case PMS_TRI15: launch_elem_t<2, 15, UPD_MODE, true, true, true>(h, a); break;
        }
        h->launches++;
        return;
    }
    switch (h->kind) {
    case PMS_TRI3: launch_elem_nn<2, 3>(h, a, upd, dof, dok, csr); break;
    case PMS_TRI6: launch_elem_nn<2, 6>(h, a, upd, dof, dok, csr); break;
    case PMS_QUA4: launch_elem_nn<2, 4>(h, a, upd, dof, dok, csr); break;
    case PMS_QUA8: launch_elem_nn<2, 8>(h, a, upd, dof, dok, csr); break;
    case PMS_QUA9: launch_elem_nn<2, 9>(h, a, upd, dof, dok, csr); break;
    case PMS_TET4: launch_elem_nn<3, 4>(h, a, upd, dof, dok, csr); break;
    case PMS_TET10: launch_elem_nn<3, 10>(h, a, upd, dof, dok, csr); break;
    case PMS_HEX8: launch_elem_nn<3, 8>(h, a, upd, dof, dok, csr); break;
    case PMS_HEX20: launch_elem_nn<3, 20>(h, a, upd, dof, dok, csr); break;
    case PMS_TRI10: launch_elem_nn<2, 10>(h, a, upd, dof, dok, csr); break;
    case PMS_TRI15: launch_elem_nn<2, 15>(h, a, upd, dof, dok, csr); break;
    }
    h->launches++;
}

ElemArgs make_args(pms_elements* h, const double* ddu) {
    ElemArgs a;
    a.ncell = h->ncell;
    a.cell0 = 0;
    a.nip = h->nip;
    a.ngauss = h->ng;
    a.thickness = h->thickness;
    a.axisym = h->axisym;
    a.coords = h->d_coords;
    a.conn = h->d_conn;
    a.cmat = h->d_cmat;
    a.mats = h->d_mats;
    a.ddu = ddu;
    a.tab = h->d_tab;
    a.sig_src = h->d_sig_b;
    a.z_src = h->d_z_b;
    a.lam_src = h->d_lam_b;
    a.el_src = h->d_el_b;
    a.sig = h->d_sig;
    a.z = h->d_z;
    a.lam = h->d_lam;
    a.el = h->d_el;
    a.fe = h->d_fe;
    a.ke = h->d_ke;
    a.ke_upper = 1;  // the gather assembly reads the upper blocks
    a.errkey = (unsigned long long*)h->d_status;
    a.bptr = h->d_bptr;
    a.cslot = h->d_cslot;
    a.crank = h->d_crank;
    a.cfirst = h->d_cfirst;
    a.order = h->d_order;
    a.ticket = h->d_ticket;
    a.next = h->d_next;
    return a;
}

// Number of public CSR values, and where the values of node A's rows start among them.
static int64_t public_nnz(const pms_elements* h) { return h->sym == PMS_SYM_FULL ? h->nnz : h->tbase[h->npoint]; }
static int64_t value_offset(const pms_elements* h, int64_t A) {
    return h->sym == PMS_SYM_FULL ? (int64_t)h->nd * h->nd * h->pat.bptr[A] : h->tbase[A];
}

template <int ND, int NN>
void launch_kk_gather_t(pms_elements* h, double* csr, const int32_t* node_prob, const uint8_t* pmode,
                        const pms::WorkQueue* q, int64_t node0, int64_t nrows, bool pub) {
    const bool tri = pub && h->sym != PMS_SYM_FULL;
    auto kern = tri ? kk_gather_kernel<ND, NN, true> : kk_gather_kernel<ND, NN, false>;
    if (h->gather_smem > 48 * 1024)
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, h->gather_smem);
    const int64_t np = q ? q->nnode : (nrows >= 0 ? nrows : h->npoint), wpb = h->gather_wpb;
    const int64_t nw = (np + GatherShape<ND, NN>::G - 1) / GatherShape<ND, NN>::G;  // warps of rows
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((nw + wpb - 1) / wpb, 148 * 32));
    kern<<<blocks, (unsigned)(32 * wpb), h->gather_smem, h->stream>>>(
        np, h->pat.nbmax, h->d_bptr, h->d_inc_ptr, h->d_inc, h->d_slot, h->d_ke, csr, node_prob, pmode,
        q ? q->nq : 0, q ? q->node_off : nullptr, q ? q->node_first : nullptr, node0, tri ? h->sym : PMS_SYM_FULL,
        h->d_kdiag, h->d_tbase);
}

// CSR gather of the block rows [node0, node0 + nrows) (nrows < 0: all), or of a work queue; pub: into
// the public layout of the values (pms_elements_set_symmetry), else the full one
void launch_kk_gather(pms_elements* h, double* csr, const int32_t* node_prob = nullptr,
                      const uint8_t* pmode = nullptr, const pms::WorkQueue* q = nullptr, int64_t node0 = 0,
                      int64_t nrows = -1, bool pub = false) {
    switch (h->kind) {
    case PMS_TRI3: launch_kk_gather_t<2, 3>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_TRI6: launch_kk_gather_t<2, 6>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_QUA4: launch_kk_gather_t<2, 4>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_QUA8: launch_kk_gather_t<2, 8>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_QUA9: launch_kk_gather_t<2, 9>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_TET4: launch_kk_gather_t<3, 4>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_TET10: launch_kk_gather_t<3, 10>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_HEX8: launch_kk_gather_t<3, 8>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_HEX20: launch_kk_gather_t<3, 20>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_TRI10: launch_kk_gather_t<2, 10>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    case PMS_TRI15: launch_kk_gather_t<2, 15>(h, csr, node_prob, pmode, q, node0, nrows, pub); break;
    }
    h->launches++;
}

void launch_f_gather(pms_elements* h, double* ff, const pms::WorkQueue* q = nullptr) {
    const int64_t n = q ? q->nnode : h->npoint;
    const int nq = q ? q->nq : 0;
    const int64_t* off = q ? q->node_off : nullptr;
    const int64_t* first = q ? q->node_first : nullptr;
    if (h->nd == 2)
        f_gather_kernel<2><<<grid_1d(n), 256, 0, h->stream>>>(n, h->d_inc_ptr, h->d_inc, h->d_fe, ff, nq, off, first);
    else
        f_gather_kernel<3><<<grid_1d(n), 256, 0, h->stream>>>(n, h->d_inc_ptr, h->d_inc, h->d_fe, ff, nq, off, first);
    h->launches++;
}

}  // namespace

namespace pms {
// Message of this thread's last refused pms_elements_create (pms_elements_last_error(NULL)).
std::string& create_error() {
    static thread_local std::string msg;
    return msg;
}

// Decodes an error key (error_key above): the element error code, cell and IP.
int decode_error(unsigned long long key, int64_t* cell, int32_t* ip) {
    if (cell) *cell = (int64_t)(((1ull << 40) - 1) - ((key >> 16) & ((1ull << 40) - 1)));
    if (ip) *ip = 255 - (int32_t)((key >> 8) & 0xff);
    return (int)(key & 0xff);
}
}  // namespace pms

extern "C" {

int pms_elements_create(const pms_mesh* mesh, const pms_material* materials, int32_t nmaterial,
                        const pms_config* config, pms_elements** out) {
    auto refuse = [](int code, const char* msg) {
        create_error() = msg;
        return code;
    };
    create_error().clear();
    if (!out) return refuse(PMS_ERR_INVALID, "out is null");
    *out = nullptr;
    if (!mesh || !materials || nmaterial < 1 || !config || !mesh->coords || !mesh->cells)
        return refuse(PMS_ERR_INVALID, "mesh, materials and config are required");
    int kind = mesh->kind;
    if (kind_nnode(kind) < 0 || kind_ndim(kind) != mesh->ndim)
        return refuse(PMS_ERR_INVALID, "unknown element kind or kind of another dimension");
    if (config->axisymmetric && mesh->ndim != 2)
        return refuse(PMS_ERR_UNSUPPORTED, "the axisymmetric idealization needs a 2D mesh");
    // plane stress: 2D linear elastic only (src/material/von_mises.rs:60-62)
    if (config->plane_stress) {
        if (mesh->ndim != 2 || config->axisymmetric)
            return refuse(PMS_ERR_UNSUPPORTED, "plane stress needs a 2D mesh without axisymmetry");
        for (int i = 0; i < nmaterial; i++)
            if (materials[i].model != PMS_LINEAR_ELASTIC)
                return refuse(PMS_ERR_UNSUPPORTED, "von Mises model does not work in plane-stress");
    }
    if (mesh->npoint < 1 || mesh->ncell < 1) return refuse(PMS_ERR_INVALID, "the mesh has no points or no cells");
    for (int i = 0; i < nmaterial; i++) {
        const pms_material& m = materials[i];
        if (m.model != PMS_LINEAR_ELASTIC && m.model != PMS_VON_MISES)
            return refuse(PMS_ERR_INVALID, "unknown stress-strain model");
        // VonMises::new (src/material/von_mises.rs:68-70)
        if (m.model == PMS_VON_MISES && !(m.z_ini > F_TOL))
            return refuse(PMS_ERR_INVALID, "von Mises initial size of the yield surface must > 1e-6");
    }
    if (mesh->cell_material) {
        for (int64_t c = 0; c < mesh->ncell; c++)
            if (mesh->cell_material[c] < 0 || mesh->cell_material[c] >= nmaterial)
                return refuse(PMS_ERR_INVALID, "cell_material names a material that does not exist");
    }
    auto* h = new pms_elements();
    h->kind = kind;
    h->nd = mesh->ndim;
    h->nc = 2 * h->nd;
    h->nn = kind_nnode(kind);
    h->npoint = mesh->npoint;
    h->ncell = mesh->ncell;
    h->ndof = h->npoint * h->nd;
    h->thickness = config->thickness > 0 ? config->thickness : 1.0;
    h->axisym = config->axisymmetric ? 1 : 0;
    std::vector<double> ksi, w;
    h->ng = integration_rule(kind, config->ngauss, ksi, w);
    if (h->ng <= 0 || h->ng > 32) {
        delete h;
        return refuse(PMS_ERR_INVALID, "requested number of integration points is not available");
    }
    h->nip = h->ncell * h->ng;
    for (int i = 0; i < nmaterial; i++) {
        const pms_material& m = materials[i];
        h->mats.push_back(make_matconst(m.model, m.young, m.poisson, m.hh, m.z_ini, config->plane_stress != 0));
    }
    // shape tables: dN[ngauss][nnode][ndim], then w[ngauss], then N[ngauss][nnode]
    h->tab.assign((size_t)h->ng * h->nn * h->nd + h->ng + (size_t)h->ng * h->nn, 0.0);
    if (pms_shape_table(kind, config->ngauss, h->tab.data(), nullptr) != PMS_OK) {
        delete h;
        return refuse(PMS_ERR_INVALID, "requested number of integration points is not available");
    }
    const char* msg = nullptr;
    if (!build_pattern(h->nd, h->nn, h->npoint, h->ncell, mesh->cells, h->pat, &msg)) {
        delete h;
        return refuse(PMS_ERR_INVALID, msg ? msg : "invalid connectivity");
    }
    h->nnz = h->pat.nblock() * h->nd * h->nd;
    // device uploads
    std::vector<int32_t> conn32((size_t)h->ncell * h->nn);
    for (size_t i = 0; i < conn32.size(); i++) conn32[i] = (int32_t)mesh->cells[i];
    bool ok = h->upload(&h->d_coords, mesh->coords, (size_t)h->npoint * h->nd) &&
              h->upload(&h->d_conn, conn32.data(), conn32.size()) &&
              h->upload(&h->d_mats, h->mats.data(), h->mats.size()) &&
              h->upload(&h->d_tab, h->tab.data(), h->tab.size());
    if (ok && mesh->cell_material) ok = h->upload(&h->d_cmat, mesh->cell_material, (size_t)h->ncell);
    ok = ok && h->alloc(&h->d_sig, (size_t)h->nip * h->nc) && h->alloc(&h->d_z, h->nip) &&
         h->alloc(&h->d_lam, h->nip) && h->alloc(&h->d_el, h->nip) &&
         h->alloc(&h->d_sig_b, (size_t)h->nip * h->nc) && h->alloc(&h->d_z_b, h->nip) &&
         h->alloc(&h->d_lam_b, h->nip) && h->alloc(&h->d_el_b, h->nip) &&
         h->alloc(&h->d_fe1, (size_t)h->nn * h->nd) &&
         h->alloc(&h->d_ke1, (size_t)h->nn * h->nd * h->nn * h->nd) &&
         h->upload(&h->d_inc_ptr, h->pat.inc_ptr.data(), h->pat.inc_ptr.size()) &&
         h->upload(&h->d_bptr, h->pat.bptr.data(), h->pat.bptr.size()) &&
         h->upload(&h->d_bcol, h->pat.bcol.data(), h->pat.bcol.size()) &&
         h->upload(&h->d_kdiag, h->pat.kdiag.data(), h->pat.kdiag.size()) &&
         h->upload(&h->d_cslot, h->pat.cslot.data(), h->pat.cslot.size()) &&
         h->upload(&h->d_crank, h->pat.crank.data(), h->pat.crank.size()) &&
         h->upload(&h->d_cfirst, h->pat.cfirst.data(), h->pat.cfirst.size()) &&
         h->upload(&h->d_order, h->pat.order.data(), h->pat.order.size()) &&
         h->alloc(&h->d_ticket, (size_t)h->npoint) && h->alloc(&h->d_next, 1) &&
         h->alloc(&h->d_ddu, h->ndof) && h->alloc(&h->d_ff, h->ndof) && h->alloc(&h->d_status, 4);
    if (!ok) {
        delete h;
        return PMS_ERR_NOMEM;
    }
    cudaMemset(h->d_status, 0, 16);
    cudaMemset(h->d_ticket, 0, (size_t)h->npoint * sizeof(int32_t));
    if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return PMS_ERR_CUDA;
    }
    h->stream = h->own_stream;
    h->smem_bytes = smem_bytes_for(h->nn, h->nd, h->ng, WPB);
    {
        // kk_gather: buffers for G = 32/nnode rows (largest block row each) per warp, up to 8
        // warps and 48 KB per block
        const int64_t row_bytes =
            (int64_t)(h->nn >= 32 ? 1 : 32 / h->nn) * std::max(h->pat.nbmax, 1) * h->nd * h->nd * 8;
        if (row_bytes > 200 * 1024) {
            delete h;
            return PMS_ERR_TOO_LARGE;
        }
        h->gather_wpb = (int)std::max<int64_t>(1, std::min<int64_t>(8, (48 * 1024) / row_bytes));
        h->gather_smem = (int)(h->gather_wpb * row_bytes);
    }
    // the state starts as LocalState::new: zero stress, elastic, zero internal variables
    init_state_kernel<<<grid_1d(h->nip), 256, 0, h->stream>>>(h->nip, h->nc, h->d_mats, h->d_cmat, h->ng, h->d_sig,
                                                              h->d_z, h->d_lam, h->d_el);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
        delete h;
        return PMS_ERR_CUDA;
    }
    *out = h;
    return PMS_OK;
}

void pms_elements_destroy(pms_elements* h) { delete h; }

int pms_elements_symmetric_jacobian(const pms_elements* h, int32_t* out) {
    if (!h || !out) return PMS_ERR_INVALID;
    bool sym = true;
    for (const MatConst& m : h->mats) sym = sym && (m.model == PMS_LINEAR_ELASTIC || m.model == PMS_VON_MISES);
    *out = sym ? 1 : 0;
    return PMS_OK;
}

int pms_elements_get_info(const pms_elements* h, pms_elements_info* o) {
    if (!h || !o) return PMS_ERR_INVALID;
    o->ndim = h->nd;
    o->kind = h->kind;
    o->nnode = h->nn;
    o->ngauss = h->ng;
    o->ncomp = h->nc;
    o->npoint = h->npoint;
    o->ncell = h->ncell;
    o->ndof = h->ndof;
    o->nip = h->nip;
    o->nnz = public_nnz(h);
    o->nblock_upper = h->pat.nupper();
    o->ncontrib = h->ncell * h->nn * h->nn;
    o->device_bytes = h->device_bytes;
    return PMS_OK;
}

int pms_elements_set_stream(pms_elements* h, void* stream) {
    if (!h) return PMS_ERR_INVALID;
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return PMS_OK;
}

// Triangle storages: the first value of each node's rows (npoint + 1).  Node A's rows hold its blocks
// on the stored side of the diagonal block and that block's own triangle (nd(nd+1)/2 entries).
static std::vector<int64_t> triangle_base(const Pattern& p, int nd, int64_t npoint, int sym) {
    const int64_t bb = (int64_t)nd * nd;
    std::vector<int64_t> tb(npoint + 1, 0);
    for (int64_t A = 0; A < npoint; A++) {
        const int64_t nb = p.bptr[A + 1] - p.bptr[A], dp = p.kdiag[A];
        tb[A + 1] = tb[A] + bb * (sym == PMS_SYM_LOWER ? dp : nb - dp - 1) + (int64_t)nd * (nd + 1) / 2;
    }
    return tb;
}

// indptr[npoint*nd + 1] / indices (either may be null) of K in the storage sym; tbase: the
// triangle_base of sym (unused for PMS_SYM_FULL).  Returns the number of values.
static int64_t fill_pattern(const Pattern& p, int nd, int64_t npoint, int sym, const std::vector<int64_t>& tbase,
                            int64_t* ipo, int32_t* ixo) {
    const int64_t nnz = sym == PMS_SYM_FULL ? p.nblock() * nd * nd : tbase[npoint];
    for (int64_t A = 0; A < npoint; A++) {
        const int64_t b0 = p.bptr[A], nb = p.bptr[A + 1] - b0;
        int64_t start = sym == PMS_SYM_FULL ? (int64_t)nd * nd * b0 : tbase[A];
        for (int i = 0; i < nd; i++) {
            const int64_t r = A * nd + i;
            if (ipo) ipo[r] = start;
            for (int64_t k = 0; k < nb; k++)
                for (int j = 0; j < nd; j++) {
                    const int64_t c = (int64_t)p.bcol[b0 + k] * nd + j;
                    if ((sym == PMS_SYM_LOWER && c > r) || (sym == PMS_SYM_UPPER && c < r)) continue;
                    if (ixo) ixo[start] = (int32_t)c;
                    start++;
                }
        }
    }
    if (ipo) ipo[npoint * nd] = nnz;
    return nnz;
}

// The CSR pattern of K in the layout sym (the device-side users inside the library take the full one).
static int csr_pattern(pms_elements* h, int64_t* indptr, int32_t* indices, int32_t mem, int sym) {
    const int nd = h->nd;
    const int64_t nnz = sym == PMS_SYM_FULL ? h->nnz : h->tbase[h->npoint];
    std::vector<int64_t> ip;
    std::vector<int32_t> ix;
    int64_t* ipo = indptr;
    int32_t* ixo = indices;
    if (mem == PMS_MEM_DEVICE) {
        ip.resize(h->ndof + 1);
        ix.resize(indices ? nnz : 0);
        ipo = ip.data();
        ixo = indices ? ix.data() : nullptr;
    }
    fill_pattern(h->pat, nd, h->npoint, sym, h->tbase, ipo, ixo);
    if (mem == PMS_MEM_DEVICE) {
        if (indptr && cudaMemcpy(indptr, ip.data(), ip.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(h, PMS_ERR_CUDA, "copy of indptr failed");
        if (indices && cudaMemcpy(indices, ix.data(), ix.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(h, PMS_ERR_CUDA, "copy of indices failed");
    }
    return PMS_OK;
}

int pms_elements_csr_pattern(pms_elements* h, int64_t* indptr, int32_t* indices, int32_t mem) {
    if (!h) return PMS_ERR_INVALID;
    return csr_pattern(h, indptr, indices, mem, h->sym);
}

int pms_elements_initialize(pms_elements* h) {
    if (!h) return PMS_ERR_INVALID;
    init_state_kernel<<<grid_1d(h->nip), 256, 0, h->stream>>>(h->nip, h->nc, h->d_mats, h->d_cmat, h->ng, h->d_sig,
                                                              h->d_z, h->d_lam, h->d_el);
    h->launches++;
    return cuda_check(h);
}

int pms_elements_reset_algorithmic(pms_elements* h) {
    if (!h) return PMS_ERR_INVALID;
    zero_lambda_kernel<<<grid_1d(h->nip), 256, 0, h->stream>>>(h->nip, h->d_lam);
    h->launches++;
    return cuda_check(h);
}

static int copy_state(pms_elements* h, bool to_backup) {
    size_t bs = (size_t)h->nip * h->nc * 8, bn = (size_t)h->nip * 8;
    double *ss = h->d_sig, *zs = h->d_z, *ls = h->d_lam, *sd = h->d_sig_b, *zd = h->d_z_b, *ld = h->d_lam_b;
    uint8_t *es = h->d_el, *ed = h->d_el_b;
    if (!to_backup) {
        std::swap(ss, sd);
        std::swap(zs, zd);
        std::swap(ls, ld);
        std::swap(es, ed);
    }
    cudaMemcpyAsync(sd, ss, bs, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(zd, zs, bn, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(ld, ls, bn, cudaMemcpyDeviceToDevice, h->stream);
    cudaMemcpyAsync(ed, es, (size_t)h->nip, cudaMemcpyDeviceToDevice, h->stream);
    return cuda_check(h);
}

int pms_elements_backup(pms_elements* h) { return h ? copy_state(h, true) : PMS_ERR_INVALID; }
int pms_elements_restore(pms_elements* h) { return h ? copy_state(h, false) : PMS_ERR_INVALID; }

static int finish_host(pms_elements* h) {
    unsigned long long key = 0;
    if (cudaMemcpyAsync(&key, h->d_status, 8, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return fail(h, PMS_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
    if (key != 0) {
        const int code = decode_error(key, &h->err_cell, &h->err_ip);
        cudaMemsetAsync(h->d_status, 0, 16, h->stream);
        switch (code) {
        case E_ZERO_SIGMA_D:
            return fail(h, PMS_ERR_ZERO_SIGMA_D,
                        "von Mises plastic update must not lead to zero sigma_d (sigma_d < 1e-10)");
        case E_ZERO_NORM_S:
            return fail(h, PMS_ERR_ZERO_NORM_S,
                        "von Mises stiffness cannot be computed with zero deviatoric norm (norm_s < 1e-10)");
        case E_JACOBIAN:
            return fail(h, PMS_ERR_JACOBIAN, "the determinant of the Jacobian must be positive");
        case E_ORDER:  // the row tickets may be left mid-count: start the next launch from zero
            cudaMemsetAsync(h->d_ticket, 0, (size_t)h->npoint * sizeof(int32_t), h->stream);
            cudaStreamSynchronize(h->stream);
            return fail(h, PMS_ERR_ORDER, "ordered assembly: a wait for an earlier cell timed out (internal error)");
        default:
            return fail(h, PMS_ERR_INVALID, "device error");
        }
    }
    return PMS_OK;
}

int pms_elements_sync(pms_elements* h) { return h ? finish_host(h) : PMS_ERR_INVALID; }

// Buffers of the gather assembly (dense F_e / K_e of every cell, incidence and slot maps), made on
// first use: the direct assembly needs none of them.
static int ensure_gather(pms_elements* h) {
    if (h->d_ke) return PMS_OK;
    const size_t ne = (size_t)h->nn * h->nd;
    const size_t nupper = (size_t)h->nn * (h->nn + 1) / 2 * h->nd * h->nd;  // upper blocks per cell
    if (!h->alloc(&h->d_fe, (size_t)h->ncell * ne) || !h->alloc(&h->d_ke, (size_t)h->ncell * nupper) ||
        !h->upload(&h->d_inc, h->pat.inc.data(), h->pat.inc.size()) ||
        !h->upload(&h->d_slot, h->pat.slot.data(), h->pat.slot.size()))
        return fail(h, PMS_ERR_NOMEM, "out of device memory for the gather assembly");
    return PMS_OK;
}

// Common path of the four batched calls.
static int run(pms_elements* h, const double* ddu, double* ff, double* csr, int mem, int upd, bool dof, bool dok) {
    if (!h || (mem != PMS_MEM_HOST && mem != PMS_MEM_DEVICE)) return PMS_ERR_INVALID;
    if (upd != UPD_NONE && !ddu) return fail(h, PMS_ERR_INVALID, "ddu is required");
    const double* d_ddu = ddu;
    double* d_ff = ff;
    double* d_csr = csr;
    if (mem == PMS_MEM_HOST) {
        if (upd != UPD_NONE) {
            cudaMemcpyAsync(h->d_ddu, ddu, (size_t)h->ndof * 8, cudaMemcpyHostToDevice, h->stream);
            d_ddu = h->d_ddu;
        }
        d_ff = ff ? h->d_ff : nullptr;
        if (csr) {
            if (!h->d_csr && !h->alloc(&h->d_csr, (size_t)h->nnz)) return fail(h, PMS_ERR_NOMEM, "out of memory");
            d_csr = h->d_csr;
        }
    }
    dof = dof && d_ff;
    dok = dok && d_csr;
    const bool direct = h->assembly == PMS_ASSEMBLY_DIRECT;
    if (!direct && (dof || dok)) {
        const int rc = ensure_gather(h);
        if (rc) return rc;
    }
    ElemArgs a = make_args(h, d_ddu);
    if (direct) {
        a.csr = d_csr;
        a.ff = d_ff;
    }
    auto timed = [h](int k, auto&& fn) {
        if (!h->timing) {
            fn();
            return;
        }
        auto e = h->event_pair();
        cudaEventRecord(e.first, h->stream);
        fn();
        cudaEventRecord(e.second, h->stream);
        h->ev_pending[k].push_back(e);
    };
    if (upd != UPD_NONE || dof || dok) timed(0, [&] { launch_elem(h, a, upd, dof, dok, direct); });
    if (dof && !direct) timed(1, [&] { launch_f_gather(h, d_ff); });
    if (mem == PMS_MEM_DEVICE || !dok || direct) {
        if (dok && !direct) timed(2, [&] { launch_kk_gather(h, d_csr, nullptr, nullptr, nullptr, 0, -1, true); });
        int rc = cuda_check(h);
        if (rc) return rc;
        if (mem == PMS_MEM_HOST) {
            if (dof) cudaMemcpyAsync(ff, d_ff, (size_t)h->ndof * 8, cudaMemcpyDeviceToHost, h->stream);
            if (dok && direct)
                cudaMemcpyAsync(csr, d_csr, (size_t)public_nnz(h) * 8, cudaMemcpyDeviceToHost, h->stream);
            return finish_host(h);
        }
        return PMS_OK;
    }
    // host CSR: gather NSLAB row slabs; each slab's values go out on the copy stream as soon as
    // the slab is written, overlapping the transfer with the later slabs (and R)
    if (!h->copy_stream) {
        if (cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess)
            return fail(h, PMS_ERR_CUDA, "stream creation failed");
        for (auto& e : h->slab_ev)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess)
                return fail(h, PMS_ERR_CUDA, "event creation failed");
    }
    constexpr int NS = pms_elements::NSLAB;
    timed(2, [&] {
        for (int k = 0; k < NS; k++) {
            const int64_t A0 = h->npoint * k / NS, A1 = h->npoint * (k + 1) / NS;
            if (A1 > A0) launch_kk_gather(h, d_csr, nullptr, nullptr, nullptr, A0, A1 - A0, true);
            cudaEventRecord(h->slab_ev[k], h->stream);
            cudaStreamWaitEvent(h->copy_stream, h->slab_ev[k], 0);
            const int64_t v0 = value_offset(h, A0), v1 = value_offset(h, A1);
            if (v1 > v0)
                cudaMemcpyAsync(csr + v0, d_csr + v0, (size_t)(v1 - v0) * 8, cudaMemcpyDeviceToHost, h->copy_stream);
        }
    });
    int rc = cuda_check(h);
    if (rc) return rc;
    if (dof) cudaMemcpyAsync(ff, d_ff, (size_t)h->ndof * 8, cudaMemcpyDeviceToHost, h->stream);
    cudaEventRecord(h->slab_ev[NS], h->copy_stream);
    cudaStreamWaitEvent(h->stream, h->slab_ev[NS], 0);
    return finish_host(h);
}

int pms_elements_update_secondary(pms_elements* h, const double* ddu, int32_t mem) {
    return run(h, ddu, nullptr, nullptr, mem, UPD_CURRENT, false, false);
}

int pms_elements_assemble_f_int(pms_elements* h, double* ff_int, int32_t mem) {
    if (!ff_int) return PMS_ERR_INVALID;
    return run(h, nullptr, ff_int, nullptr, mem, UPD_NONE, true, false);
}

int pms_elements_assemble_kk(pms_elements* h, double* csr_values, int32_t mem) {
    if (!csr_values) return PMS_ERR_INVALID;
    return run(h, nullptr, nullptr, csr_values, mem, UPD_NONE, false, true);
}

int pms_elements_update_and_assemble(pms_elements* h, const double* ddu, double* ff_int, double* csr_values,
                                     int32_t mem) {
    return run(h, ddu, ff_int, csr_values, mem, UPD_BACKUP, ff_int != nullptr, csr_values != nullptr);
}

static int one_cell(pms_elements* h, int64_t cell, bool dof, bool dok) {
    if (!h || cell < 0 || cell >= h->ncell) return PMS_ERR_INVALID;
    ElemArgs a = make_args(h, nullptr);
    a.ncell = 1;
    a.cell0 = cell;
    a.fe = h->d_fe1;  // dense outputs of this one cell
    a.ke = h->d_ke1;
    a.ke_upper = 0;  // full matrix for the caller
    a.ke_cell0 = cell;
    launch_elem(h, a, UPD_NONE, dof, dok, false);
    int rc = cuda_check(h);
    if (rc) return rc;
    return finish_host(h);
}

int pms_element_calc_f_int(pms_elements* h, int64_t cell, double* f) {
    if (!f) return PMS_ERR_INVALID;
    int rc = one_cell(h, cell, true, false);
    if (rc) return rc;
    if (cudaMemcpy(f, h->d_fe1, (size_t)h->nn * h->nd * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(h, PMS_ERR_CUDA, "copy failed");
    return PMS_OK;
}

int pms_element_calc_jacobian(pms_elements* h, int64_t cell, double* kk) {
    if (!kk) return PMS_ERR_INVALID;
    int rc = one_cell(h, cell, false, true);
    if (rc) return rc;
    const int64_t ne = h->nn * h->nd;
    if (cudaMemcpy(kk, h->d_ke1, (size_t)(ne * ne) * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(h, PMS_ERR_CUDA, "copy failed");
    return PMS_OK;
}

int pms_elements_get_state(pms_elements* h, double* sig, double* ivs, uint8_t* elastic) {
    if (!h) return PMS_ERR_INVALID;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(h, PMS_ERR_CUDA, "sync failed");
    const int64_t n = h->nip;
    std::vector<double> s((size_t)n * h->nc), z(n), l(n);
    std::vector<uint8_t> e(n);
    cudaMemcpy(s.data(), h->d_sig, s.size() * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(z.data(), h->d_z, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(l.data(), h->d_lam, n * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(e.data(), h->d_el, n, cudaMemcpyDeviceToHost);
    for (int64_t i = 0; i < n; i++) {
        if (sig)
            for (int c = 0; c < h->nc; c++) sig[i * h->nc + c] = s[(size_t)c * n + i];
        if (ivs) {
            ivs[2 * i] = z[i];
            ivs[2 * i + 1] = l[i];
        }
        if (elastic) elastic[i] = e[i];
    }
    return cuda_check(h);
}

int pms_elements_set_state(pms_elements* h, const double* sig, const double* ivs, const uint8_t* elastic) {
    if (!h || !sig || !ivs || !elastic) return PMS_ERR_INVALID;
    const int64_t n = h->nip;
    std::vector<double> s((size_t)n * h->nc), z(n), l(n);
    for (int64_t i = 0; i < n; i++) {
        for (int c = 0; c < h->nc; c++) s[(size_t)c * n + i] = sig[i * h->nc + c];
        z[i] = ivs[2 * i];
        l[i] = ivs[2 * i + 1];
    }
    cudaStreamSynchronize(h->stream);
    cudaMemcpy(h->d_sig, s.data(), s.size() * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_z, z.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_lam, l.data(), n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(h->d_el, elastic, n, cudaMemcpyHostToDevice);
    return cuda_check(h);
}

const char* pms_elements_last_error(const pms_elements* h) { return h ? h->last_error.c_str() : create_error().c_str(); }

int pms_elements_error_location(const pms_elements* h, int64_t* cell, int32_t* ip) {
    if (!h) return PMS_ERR_INVALID;
    if (cell) *cell = h->err_cell;
    if (ip) *ip = h->err_ip;
    return PMS_OK;
}

int64_t pms_elements_launch_count(const pms_elements* h) { return h ? h->launches : 0; }

int pms_elements_set_assembly(pms_elements* h, int32_t mode) {
    if (!h || (mode != PMS_ASSEMBLY_DIRECT && mode != PMS_ASSEMBLY_GATHER)) return PMS_ERR_INVALID;
    if (mode == PMS_ASSEMBLY_DIRECT && h->sym != PMS_SYM_FULL)
        return fail(h, PMS_ERR_UNSUPPORTED, "the direct assembly writes both triangles of K");
    h->assembly = mode;
    return PMS_OK;
}

int pms_elements_set_symmetry(pms_elements* h, int32_t sym) {
    if (!h || (sym != PMS_SYM_FULL && sym != PMS_SYM_LOWER && sym != PMS_SYM_UPPER)) return PMS_ERR_INVALID;
    if (sym != PMS_SYM_FULL && h->assembly == PMS_ASSEMBLY_DIRECT)
        return fail(h, PMS_ERR_UNSUPPORTED, "the direct assembly writes both triangles of K");
    if (sym != PMS_SYM_FULL) {
        std::vector<int64_t> tb = triangle_base(h->pat, h->nd, h->npoint, sym);
        if (!h->d_tbase && !h->alloc(&h->d_tbase, (size_t)h->npoint + 1))
            return fail(h, PMS_ERR_NOMEM, "out of device memory");
        if (cudaMemcpy(h->d_tbase, tb.data(), tb.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess)
            return fail(h, PMS_ERR_CUDA, "copy of the triangle offsets failed");
        h->tbase.swap(tb);
    }
    h->sym = sym;
    return PMS_OK;
}

int pms_elements_set_timing(pms_elements* h, int32_t on) {
    if (!h) return PMS_ERR_INVALID;
    h->timing = on != 0;
    return PMS_OK;
}

int pms_elements_kernel_times(pms_elements* h, double* ms, int64_t* counts) {
    if (!h) return PMS_ERR_INVALID;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(h, PMS_ERR_CUDA, "sync failed");
    for (int k = 0; k < 3; k++) {
        double tot = 0.0;
        for (auto& e : h->ev_pending[k]) {
            float t = 0.f;
            cudaEventElapsedTime(&t, e.first, e.second);
            tot += t;
            h->ev_pool.push_back(e);
        }
        if (ms) ms[k] = tot;
        if (counts) counts[k] = (int64_t)h->ev_pending[k].size();
        h->ev_pending[k].clear();
    }
    return cuda_check(h);
}

int pms_mesh_assembly_maps(const pms_mesh* mesh, int16_t* cslot, int32_t* crank, uint32_t* cfirst, int32_t* order) {
    if (!mesh || !mesh->cells || kind_nnode(mesh->kind) < 0 || kind_ndim(mesh->kind) != mesh->ndim)
        return PMS_ERR_INVALID;
    Pattern p;
    const char* msg = nullptr;
    if (!build_pattern(mesh->ndim, kind_nnode(mesh->kind), mesh->npoint, mesh->ncell, mesh->cells, p, &msg))
        return PMS_ERR_INVALID;
    if (cslot) std::memcpy(cslot, p.cslot.data(), p.cslot.size() * sizeof(int16_t));
    if (crank) std::memcpy(crank, p.crank.data(), p.crank.size() * sizeof(int32_t));
    if (cfirst) std::memcpy(cfirst, p.cfirst.data(), p.cfirst.size() * sizeof(uint32_t));
    if (order) std::memcpy(order, p.order.data(), p.order.size() * sizeof(int32_t));
    return PMS_OK;
}

int pms_shape_table(int32_t kind, int32_t ngauss, double* tab, int32_t* ngauss_out) {
    const int nn = kind_nnode(kind), nd = kind_ndim(kind);
    if (nn < 0) return PMS_ERR_INVALID;
    double ksi[3 * 27], w[27];
    const int ng = integration_rule_into(kind, ngauss, ksi, w);
    if (ng <= 0) return PMS_ERR_INVALID;
    if (ngauss_out) *ngauss_out = ng;
    if (!tab) return PMS_OK;
    double N[20], dN[60];
    for (int p = 0; p < ng; p++) {
        shape_eval(kind, &ksi[3 * p], N, dN);
        for (int m = 0; m < nn; m++)
            for (int j = 0; j < nd; j++) tab[(p * nn + m) * nd + j] = dN[m * nd + j];
        tab[(size_t)ng * nn * nd + p] = w[p];
        for (int m = 0; m < nn; m++) tab[(size_t)ng * nn * nd + ng + p * nn + m] = N[m];
    }
    return PMS_OK;
}

int pms_mesh_csr_pattern_sym(const pms_mesh* mesh, int32_t sym, int64_t* indptr, int32_t* indices, int64_t* nnz) {
    if (!mesh || !mesh->cells || kind_nnode(mesh->kind) < 0 || kind_ndim(mesh->kind) != mesh->ndim ||
        (sym != PMS_SYM_FULL && sym != PMS_SYM_LOWER && sym != PMS_SYM_UPPER))
        return PMS_ERR_INVALID;
    Pattern p;
    const char* msg = nullptr;
    const int nd = mesh->ndim;
    if (!build_pattern(nd, kind_nnode(mesh->kind), mesh->npoint, mesh->ncell, mesh->cells, p, &msg))
        return PMS_ERR_INVALID;
    const std::vector<int64_t> tb =
        sym == PMS_SYM_FULL ? std::vector<int64_t>() : triangle_base(p, nd, mesh->npoint, sym);
    const int64_t total = fill_pattern(p, nd, mesh->npoint, sym, tb, indptr, indices);
    if (nnz) *nnz = total;
    return PMS_OK;
}

int pms_mesh_csr_pattern(const pms_mesh* mesh, int64_t* indptr, int32_t* indices, int64_t* nnz) {
    return pms_mesh_csr_pattern_sym(mesh, PMS_SYM_FULL, indptr, indices, nnz);
}

}  // extern "C"

// ------------------------------------------------------------------------------------------
// Internal interface used by the batched solver (pms_internal.h).
namespace pms {

ElementsView elements_view(pms_elements* h) {
    ElementsView v;
    v.nd = h->nd;
    v.nn = h->nn;
    v.ng = h->ng;
    v.npoint = h->npoint;
    v.ncell = h->ncell;
    v.ndof = h->ndof;
    v.nnz = h->nnz;
    v.d_bptr = h->d_bptr;
    v.d_bcol = h->d_bcol;
    v.d_kdiag = h->d_kdiag;
    v.stream = h->stream;
    return v;
}

std::mutex& device_mutex() {
    static std::mutex m;
    return m;
}

int elements_device_pattern(pms_elements* h, const int64_t** indptr, const int32_t** indices) {
    if (!h->d_indptr) {
        if (!h->alloc(&h->d_indptr, (size_t)h->ndof + 1) || !h->alloc(&h->d_indices, (size_t)h->nnz))
            return fail(h, PMS_ERR_NOMEM, "out of device memory for the CSR pattern");
        int rc = csr_pattern(h, h->d_indptr, h->d_indices, PMS_MEM_DEVICE, PMS_SYM_FULL);
        if (rc) return rc;
    }
    *indptr = h->d_indptr;
    *indices = h->d_indices;
    return PMS_OK;
}

int elements_run_modes(pms_elements* h, const int32_t* cell_prob, const int32_t* node_prob, const uint8_t* pmode,
                       const double* ddu, double* ff, double* csr, const WorkQueue* queue,
                       unsigned long long* prob_err) {
    ElemArgs a = make_args(h, ddu);
    a.cell_prob = cell_prob;
    a.pmode = pmode;
    a.prob_err = prob_err;
    if (queue) {
        if (queue->nq <= 0 || queue->ncell <= 0) return PMS_OK;  // nothing queued
        a.ncell = queue->ncell;
        a.nq = queue->nq;
        a.q_off = queue->cell_off;
        a.q_first = queue->cell_first;
    }
    a.csr = csr;  // direct assembly: rows of problems outside the pass are left as they are
    a.ff = ff;
    (void)node_prob;
    launch_elem(h, a, UPD_MODE, true, true, true);
    return cuda_check(h);
}

int elements_status(pms_elements* h) { return finish_host(h); }

namespace graph_pass {
// Launch shape of the per-problem-mode element kernel (as launch_elem_t<..., UPD_MODE, F, K, CSR>).
struct ElemLaunchShape {
    const void* func = nullptr;
    unsigned grid = 1, block = 128;
    int smem = 0;
};

template <int NN, int LPC>
ElemLaunchShape mode_shape_2d(const ElemArgs& a) {
    constexpr int CPW = 32 / LPC;
    auto kern = element2d_kernel<NN, LPC, UPD_MODE, true, true, true>;
    const int smem = smem2_bytes(NN, a.ngauss, CPW, true);
    allow_dynamic_smem((const void*)kern);
    cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    int64_t blocks = ((a.ncell + CPW - 1) / CPW + WPB2 - 1) / WPB2;
    blocks = std::min<int64_t>(blocks, resident_blocks((const void*)kern, smem, WPB2 * 32));
    ElemLaunchShape r;
    r.func = (const void*)kern;
    r.grid = (unsigned)std::max<int64_t>(blocks, 1);
    r.block = WPB2 * 32;
    r.smem = smem;
    return r;
}

template <int ND, int NN>
ElemLaunchShape mode_shape(pms_elements* h, const ElemArgs& a) {
    if constexpr (ND == 2 && fits_2d<NN>()) {
        if (a.ngauss <= NG2_MAX) {
            if constexpr (packed_layout<NN>())
                if (a.ngauss <= lanes_packed<NN>()) return mode_shape_2d<NN, lanes_packed<NN>()>(a);
            return mode_shape_2d<NN, 16>(a);
        }
    }
    auto kern = element_kernel<ND, NN, UPD_MODE, true, true, true>;
    allow_dynamic_smem((const void*)kern);
    int64_t blocks = (a.ncell + cells_per_block(NN) - 1) / cells_per_block(NN);
    blocks = std::min<int64_t>(blocks, resident_blocks((const void*)kern, h->smem_bytes));
    ElemLaunchShape r;
    r.func = (const void*)kern;
    r.grid = (unsigned)std::max<int64_t>(blocks, 1);
    r.block = WPB * 32;
    r.smem = h->smem_bytes;
    return r;
}
}  // namespace graph_pass

int elements_graph_pass(pms_elements* h, cudaGraph_t g, cudaGraphNode_t dep, cudaGraphNode_t* last,
                        const int32_t* cell_prob, const uint8_t* pmode, const double* ddu, double* ff, double* csr,
                        unsigned long long* prob_err) {
    ElemArgs a = make_args(h, ddu);
    a.cell_prob = cell_prob;
    a.pmode = pmode;
    a.prob_err = prob_err;
    a.csr = csr;
    a.ff = ff;
    using namespace graph_pass;
    ElemLaunchShape sh;
    switch (h->kind) {
    case PMS_TRI3: sh = mode_shape<2, 3>(h, a); break;
    case PMS_TRI6: sh = mode_shape<2, 6>(h, a); break;
    case PMS_QUA4: sh = mode_shape<2, 4>(h, a); break;
    case PMS_QUA8: sh = mode_shape<2, 8>(h, a); break;
    case PMS_QUA9: sh = mode_shape<2, 9>(h, a); break;
    case PMS_TET4: sh = mode_shape<3, 4>(h, a); break;
    case PMS_TET10: sh = mode_shape<3, 10>(h, a); break;
    case PMS_HEX8: sh = mode_shape<3, 8>(h, a); break;
    case PMS_HEX20: sh = mode_shape<3, 20>(h, a); break;
    case PMS_TRI10: sh = mode_shape<2, 10>(h, a); break;
    case PMS_TRI15: sh = mode_shape<2, 15>(h, a); break;
    default: return fail(h, PMS_ERR_INVALID, "unknown element kind");
    }
    cudaMemsetParams mp = {};
    mp.dst = (void*)h->d_next;
    mp.value = 0;
    mp.elementSize = 4;
    mp.width = 2;  // the 8-byte counter
    mp.height = 1;
    mp.pitch = 0;
    cudaGraphNode_t nm, nk;
    if (cudaGraphAddMemsetNode(&nm, g, dep ? &dep : nullptr, dep ? 1 : 0, &mp) != cudaSuccess)
        return fail(h, PMS_ERR_CUDA, "graph memset node failed");
    void* args[] = {&a};
    cudaKernelNodeParams kp = {};
    kp.func = (void*)sh.func;
    kp.gridDim = dim3(sh.grid);
    kp.blockDim = dim3(sh.block);
    kp.sharedMemBytes = (unsigned)sh.smem;
    kp.kernelParams = args;
    if (cudaGraphAddKernelNode(&nk, g, &nm, 1, &kp) != cudaSuccess)
        return fail(h, PMS_ERR_CUDA, "graph element node failed");
    h->launches++;
    *last = nk;
    return PMS_OK;
}

}  // namespace pms

// ------------------------------------------------------------------------------------------
// Element matrices without any device allocation.
//
// Some callers cannot call cudaMalloc: a host program that runs inside another framework's
// fixed device-memory budget (the framework owns every allocation), a real-time loop where an
// allocation would stall or synchronise the device, or a foreign-language caller (for example a
// Rust element loop behind an FFI) that has no CUDA allocator at all.  For them this entry point
// takes host inputs and host outputs and keeps everything it needs on the device in one
// file-scope array of fixed size, so it never allocates.  Limit: NOALLOC_SCRATCH_BYTES per
// device, held by every GPU that loads this library until the process exits; a call whose cells
// do not fit is rejected (the largest batch that fits is reported back).  All calls share the
// array and it keeps the last call's contents, so calls that overlap on the GPU (two host
// threads, or two streams without ordering) race: serialise them.  The first call on a device
// looks up the array's device address (cudaGetSymbolAddress) for that device; make that first
// call before any stream capture.
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(16) << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
void* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {nullptr};

__global__ void iota_kernel(int64_t n, int32_t* out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)i;
}

inline size_t up256(size_t b) { return (b + 255) & ~size_t(255); }

struct NoallocLayout {
    size_t status, tab, mat, coords, conn, sig, z, lam, el, fe, ke, total;
};

NoallocLayout noalloc_layout(int nn, int nd, int ng, int64_t ncell, bool want_f, bool want_k) {
    const int nc = 2 * nd, ne = nn * nd;
    const int64_t nip = ncell * ng;
    NoallocLayout L;
    size_t o = 0;
    L.status = o; o += 256;
    L.tab = o; o += up256(sizeof(double) * ((size_t)ng * nn * nd + ng));
    L.mat = o; o += up256(sizeof(MatConst));
    L.coords = o; o += up256(sizeof(double) * (size_t)ncell * nn * nd);
    L.conn = o; o += up256(sizeof(int32_t) * (size_t)ncell * nn);
    L.sig = o; o += up256(sizeof(double) * (size_t)nip * nc);
    L.z = o; o += up256(sizeof(double) * (size_t)nip);
    L.lam = o; o += up256(sizeof(double) * (size_t)nip);
    L.el = o; o += up256((size_t)nip);
    L.fe = o; o += want_f ? up256(sizeof(double) * (size_t)ncell * nn * nd) : 0;
    L.ke = o; o += want_k ? up256(sizeof(double) * (size_t)ncell * ne * ne) : 0;
    L.total = o;
    return L;
}

template <int ND, int NN, bool DOF, bool DOK>
void noalloc_launch_t(const ElemArgs& a, int smem, cudaStream_t st) {
    if constexpr (ND == 2 && fits_2d<NN>()) {
        if (a.ngauss <= NG2_MAX) {
            launch_elem2d_t<NN, UPD_NONE, DOF, DOK, false>(a, st, false);
            return;
        }
    }
    auto kern = element_kernel<ND, NN, UPD_NONE, DOF, DOK, false>;
    allow_dynamic_smem((const void*)kern);
    kern<<<(unsigned)((a.ncell + cells_per_block(NN) - 1) / cells_per_block(NN)), WPB * 32, smem, st>>>(a);
}

template <int ND, int NN>
void noalloc_launch(const ElemArgs& a, bool dof, bool dok, int smem, cudaStream_t st) {
    if (dof && dok) noalloc_launch_t<ND, NN, true, true>(a, smem, st);
    else if (dof) noalloc_launch_t<ND, NN, true, false>(a, smem, st);
    else noalloc_launch_t<ND, NN, false, true>(a, smem, st);
}

}  // namespace

extern "C" int pms_element_calc_noalloc(int32_t kind, int32_t ngauss, double thickness, const pms_material* mat,
                                        int64_t ncell, const double* X, const double* sig, const double* ivs,
                                        const uint8_t* elastic, double* f, double* kk, int64_t* max_cells,
                                        void* stream) {
    if (kind_nnode(kind) < 0 || !mat || ncell < 0 || (!f && !kk)) return PMS_ERR_INVALID;
    if (mat->model != PMS_LINEAR_ELASTIC && mat->model != PMS_VON_MISES) return PMS_ERR_INVALID;
    if (mat->model == PMS_VON_MISES && !(mat->z_ini > F_TOL)) return PMS_ERR_INVALID;
    const int nn = kind_nnode(kind), nd = kind_ndim(kind), nc = 2 * nd;
    // integration rule and shape table on the stack (no heap): at most 27 x 20 x 3 + 27 doubles
    double ksi_buf[27 * 3], w_buf[27];
    const int ng = integration_rule_into(kind, ngauss, ksi_buf, w_buf);
    if (ng <= 0 || ng > 27) return PMS_ERR_INVALID;
    // largest batch that fits (binary search on the layout size)
    {
        int64_t lo = 0, hi = (int64_t)(NOALLOC_SCRATCH_BYTES / 64);
        while (lo < hi) {
            const int64_t mid = (lo + hi + 1) / 2;
            if (noalloc_layout(nn, nd, ng, mid, f != nullptr, kk != nullptr).total <= NOALLOC_SCRATCH_BYTES)
                lo = mid;
            else
                hi = mid - 1;
        }
        if (max_cells) *max_cells = lo;
        if (ncell > lo) return PMS_ERR_TOO_LARGE;  // batch larger than the fixed scratch: split it
    }
    if (ncell == 0) return PMS_OK;
    if (!X || !sig || !ivs || !elastic) return PMS_ERR_INVALID;
    // device address of the scratch array, looked up once per device
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return PMS_ERR_CUDA;
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return PMS_ERR_CUDA;
        g_noalloc_addr[dev] = p;
    }
    unsigned char* base = (unsigned char*)g_noalloc_addr[dev];
    cudaStream_t st = (cudaStream_t)stream;
    const NoallocLayout L = noalloc_layout(nn, nd, ng, ncell, f != nullptr, kk != nullptr);
    const int64_t nip = ncell * ng;
    // shape table
    double tab[27 * 20 * 3 + 27];
    {
        double N[20], dN[60];
        for (int p = 0; p < ng; p++) {
            shape_eval(kind, &ksi_buf[3 * p], N, dN);
            for (int m = 0; m < nn; m++)
                for (int j = 0; j < nd; j++) tab[(p * nn + m) * nd + j] = dN[m * nd + j];
            tab[ng * nn * nd + p] = w_buf[p];
        }
    }
    const MatConst mc = make_matconst(mat->model, mat->young, mat->poisson, mat->hh, mat->z_ini);
    const int tab_len = ng * nn * nd + ng;
    bool ok = cudaMemsetAsync(base + L.status, 0, 16, st) == cudaSuccess;  // status must start at zero
    ok = ok && cudaMemcpyAsync(base + L.tab, tab, sizeof(double) * tab_len, cudaMemcpyHostToDevice, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(base + L.mat, &mc, sizeof(MatConst), cudaMemcpyHostToDevice, st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(base + L.coords, X, sizeof(double) * (size_t)ncell * nn * nd, cudaMemcpyHostToDevice,
                               st) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(base + L.sig, sig, sizeof(double) * (size_t)nip * nc, cudaMemcpyHostToDevice, st) ==
                   cudaSuccess;
    ok = ok && cudaMemcpyAsync(base + L.z, ivs, sizeof(double) * (size_t)nip, cudaMemcpyHostToDevice, st) ==
                   cudaSuccess;
    ok = ok && cudaMemcpyAsync(base + L.lam, ivs + nip, sizeof(double) * (size_t)nip, cudaMemcpyHostToDevice, st) ==
                   cudaSuccess;
    ok = ok && cudaMemcpyAsync(base + L.el, elastic, (size_t)nip, cudaMemcpyHostToDevice, st) == cudaSuccess;
    if (!ok) return PMS_ERR_CUDA;
    iota_kernel<<<(unsigned)std::min<int64_t>((ncell * nn + 255) / 256, 1024), 256, 0, st>>>(
        ncell * nn, (int32_t*)(base + L.conn));
    ElemArgs a;
    a.ncell = ncell;
    a.cell0 = 0;
    a.nip = nip;
    a.ngauss = ng;
    a.thickness = thickness > 0 ? thickness : 1.0;
    a.coords = (const double*)(base + L.coords);
    a.conn = (const int32_t*)(base + L.conn);
    a.cmat = nullptr;
    a.mats = (const MatConst*)(base + L.mat);
    a.ddu = nullptr;
    a.tab = (const double*)(base + L.tab);
    a.sig_src = nullptr;
    a.z_src = nullptr;
    a.lam_src = nullptr;
    a.el_src = nullptr;
    a.sig = (double*)(base + L.sig);
    a.z = (double*)(base + L.z);
    a.lam = (double*)(base + L.lam);
    a.el = (uint8_t*)(base + L.el);
    a.fe = (double*)(base + L.fe);
    a.ke = (double*)(base + L.ke);
    a.errkey = (unsigned long long*)(base + L.status);
    const int smem = smem_bytes_for(nn, nd, ng, WPB);
    const bool dof = f != nullptr, dok = kk != nullptr;
    switch (kind) {
    case PMS_TRI3: noalloc_launch<2, 3>(a, dof, dok, smem, st); break;
    case PMS_TRI6: noalloc_launch<2, 6>(a, dof, dok, smem, st); break;
    case PMS_QUA4: noalloc_launch<2, 4>(a, dof, dok, smem, st); break;
    case PMS_QUA8: noalloc_launch<2, 8>(a, dof, dok, smem, st); break;
    case PMS_QUA9: noalloc_launch<2, 9>(a, dof, dok, smem, st); break;
    case PMS_TET4: noalloc_launch<3, 4>(a, dof, dok, smem, st); break;
    case PMS_TET10: noalloc_launch<3, 10>(a, dof, dok, smem, st); break;
    case PMS_HEX8: noalloc_launch<3, 8>(a, dof, dok, smem, st); break;
    case PMS_HEX20: noalloc_launch<3, 20>(a, dof, dok, smem, st); break;
    case PMS_TRI10: noalloc_launch<2, 10>(a, dof, dok, smem, st); break;
    case PMS_TRI15: noalloc_launch<2, 15>(a, dof, dok, smem, st); break;
    }
    if (cudaGetLastError() != cudaSuccess) return PMS_ERR_CUDA;
    const int ne = nn * nd;
    if (dof && cudaMemcpyAsync(f, base + L.fe, sizeof(double) * (size_t)ncell * ne, cudaMemcpyDeviceToHost, st) !=
                   cudaSuccess)
        return PMS_ERR_CUDA;
    if (dok && cudaMemcpyAsync(kk, base + L.ke, sizeof(double) * (size_t)ncell * ne * ne, cudaMemcpyDeviceToHost,
                               st) != cudaSuccess)
        return PMS_ERR_CUDA;
    unsigned long long key = 0;
    if (cudaMemcpyAsync(&key, base + L.status, 8, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return PMS_ERR_CUDA;
    switch (decode_error(key, nullptr, nullptr)) {
    case 0: return PMS_OK;
    case E_ZERO_NORM_S: return PMS_ERR_ZERO_NORM_S;
    case E_JACOBIAN: return PMS_ERR_JACOBIAN;
    case E_ZERO_SIGMA_D: return PMS_ERR_ZERO_SIGMA_D;
    default: return PMS_ERR_INVALID;
    }
}
