// pms_internal.h -- C++ interface between the element handle (pms_elements.cu) and the batched
// Newton/PCG solver (pms_solver.cu).  Not part of the C ABI.
#pragma once
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

#include "../../include/pms.h"

namespace pms {

// Serialises CUDA graph capture against device allocation and release across host threads: a
// cudaFree (which synchronises the device) issued by one thread while another thread captures a
// graph would invalidate that capture.  Handles in different threads (served batches) take it
// around cudaMalloc/cudaFree and around each capture.
std::mutex& device_mutex();

struct ElementsView {
    int nd, nn, ng;
    int64_t npoint, ncell, ndof, nnz;
    const int64_t* d_bptr;   // block-row pointers (npoint + 1)
    const int32_t* d_bcol;   // block columns (node ids, sorted in each block row)
    const int32_t* d_kdiag;  // position of the diagonal block in each block row
    cudaStream_t stream;
};

ElementsView elements_view(pms_elements* h);

// Device CSR pattern of K (allocated by the handle on first use, kept until destroy).
int elements_device_pattern(pms_elements* h, const int64_t** indptr, const int32_t** indices);

// Work queue of a batched element pass: the cell ranges and node ranges of the problems that take
// part (device arrays; range k covers off[k] .. off[k+1]-1 of the queue, starting at first[k]).
struct WorkQueue {
    int32_t nq = 0;
    int64_t ncell = 0, nnode = 0;  // queued cells and nodes (off[nq])
    const int64_t* cell_off = nullptr;
    const int64_t* cell_first = nullptr;
    const int64_t* node_off = nullptr;
    const int64_t* node_first = nullptr;
};

// One launch of the element kernel in per-problem mode (0 skip, 1 step start, 2 update) followed by
// the F_int and CSR gathers (the CSR rows of mode-0 problems are left as they are); all pointers
// are device pointers on the handle's stream.  With a queue, only its cells and nodes are visited
// (every queued problem must have a non-zero mode); F_int rows outside the queue are left as they are.
// prob_err (device, nullable): per problem, the key of the element error that problem would report
// (atomicMax; the caller zeroes it before the launch; decode with decode_error).
int elements_run_modes(pms_elements* h, const int32_t* cell_prob, const int32_t* node_prob, const uint8_t* pmode,
                       const double* ddu, double* ff, double* csr, const WorkQueue* queue = nullptr,
                       unsigned long long* prob_err = nullptr);

// Adds to graph g (after dep, if not null) a memset node that zeroes the element pass's in-order work
// counter and the node of the per-problem-mode element kernel over every cell (direct assembly into
// csr and ff; cells of problems whose mode is 0 are skipped; per-problem error keys in prob_err);
// *last receives the kernel node.  The same kernel and arithmetic as elements_run_modes.
int elements_graph_pass(pms_elements* h, cudaGraph_t g, cudaGraphNode_t dep, cudaGraphNode_t* last,
                        const int32_t* cell_prob, const uint8_t* pmode, const double* ddu, double* ff, double* csr,
                        unsigned long long* prob_err);

// Element error key -> element error code (internal E_* value), cell and IP.
int decode_error(unsigned long long key, int64_t* cell, int32_t* ip);

// Status of the last launches (waits for the handle's stream).
int elements_status(pms_elements* h);

}  // namespace pms
