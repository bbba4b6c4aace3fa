// Device-side plan and per-factorization state of the multifrontal LDL^T.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace b200ldl {

// Immutable per-pattern data uploaded once after the symbolic phase. All
// arrays are indexed by supernode id (the reference's node numbering) unless
// stated otherwise.
struct DevPlan {
  int n;
  int num_nodes;
  const int* ns;            // [nn] pivot columns of the supernode
  const int* nc;            // [nn] symbolic contribution rows
  const int* var_ptr;       // [nn+1] into node_to_var
  const int* node_to_var;   // [n] original numbering
  const int* cptr;          // [nn+1] into contrib_rows / cmap
  const int* contrib_rows;  // original numbering
  const int* cmap;          // static position of each contrib row in the parent front
  const int* kid_ptr;       // [nn+1]
  const int* kids;          // children, reference order
  const int64_t* scat_ptr;  // [nn+1] into the scatter lists
  const int* scat_csr;      // CSR value index
  const int* scat_row;      // static row position (own var j, or ns + contrib index)
  const int* scat_col;      // own column j
};

// A front too large for shared memory, registered by the level kernel and
// factored by the cluster panel / tiled update kernels.
struct BigFront {
  int node, f, fs, ns, nd_in, nc;
  int k, ncand, kstart, kw;
  int state;  // 0 active, 1 finished after the pending update, 2 done
  int npos, nneg;
  int pad;
  long long ioff;  // front variables (fv[f], orig[f]) in the int pool
  long long doff;  // the front F (f x f, column-major) in the double pool
  long long woff;  // the panel's W columns (f x kBigPanelMax) in the double pool
  double flops;
};

constexpr int kBigPanelMax = 32;

// Mutable state of one factorization (device memory).
struct DevState {
  int* f;       // [nn] front size at run time
  int* fs;      // [nn] fully summed (candidates)
  int* npiv;    // [nn]
  int* ndel;    // [nn] delayed to the parent
  int64_t* fv_off;  // [nn] into ivars: fv[f] then orig[f]
  int64_t* L_off;   // [nn] into dpool, L is f x npiv, ld = L_ld
  int* L_ld;        // [nn]
  int64_t* cb_off;  // [nn] into dpool, lower (f-npiv)^2 block, ld = cb_ld
  int* cb_ld;       // [nn]
  int* ivars;       // int pool
  double* dpool;    // double pool (factors, contribution blocks, big fronts)
  unsigned long long* used;  // [3]: ints used, doubles used, update rows used
  unsigned long long icap, dcap;
  int64_t* u_off;   // [nn] into the solve's update-vector pool (units of rows)
  int* err;         // [4]: [0] overflow flag, [1] node of first error
  int* inertia;     // [2] pos, neg
  double* flops;    // [1] executed factor flops (accumulated)
  BigFront* big;    // [nn] big fronts of the current level
  int* big_meta;    // [4]: count, max f, max fs, unused
  long long* tile_ptr;  // [nn+1] update tiles per big front (prefix)
};

struct FactorParams {
  double ustab;
  double pivot_tol;
  int cholesky;
};

// Largest front factored entirely in shared memory (fp64, ld = f | 1).
constexpr int kSmemFrontMax = 144;
constexpr int kFactorThreads = 256;

void launch_factor_level(const DevPlan& p, const DevState& s,
                         const int* level_nodes, int count,
                         const FactorParams& prm, cudaStream_t stream,
                         const double* vals, const double* diag);
cudaError_t configure_factor_kernels();
size_t factor_smem_bytes();

// Big-front pipeline for one level (see big.cu). `maxkids` is the largest
// number of children among the level's supernodes.
struct BigLevelInfo {
  int count, max_f, max_fs;
};
cudaError_t launch_big_level(const DevPlan& p, const DevState& s, const BigLevelInfo& info,
                      int maxkids, const FactorParams& prm, const double* vals,
                      const double* diag, cudaStream_t stream);
cudaError_t configure_big_kernels();

constexpr int kSolveThreads = 256;
// Front vectors of the solve live in shared memory up to this front size.
constexpr int kSolveSmemFront = 12288;

void launch_forward_level(const DevPlan& p, const DevState& s,
                          const int* level_nodes, int count, double* x,
                          int ldx, int nrhs, double* upool, int fmax,
                          cudaStream_t stream);
void launch_backward_level(const DevPlan& p, const DevState& s,
                           const int* level_nodes, int count, double* x,
                           int ldx, int nrhs, int fmax, cudaStream_t stream);
cudaError_t configure_solve_kernels();

}  // namespace b200ldl
