// Device-side plan and per-factorization state of the multifrontal LDL^T.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <utility>
#include <vector>

struct b200ldl_assembly;  // the assembly plan of the C ABI (assembly.cu)

namespace b200ldl {

// Work counters accumulated on the device per factorization.
constexpr int kWork = 8;

// Kernel classes timed by the optional profiler.
enum ProfPhase : int {
  kPhFront = 0,     // per-level front kernels (assembly + factor in shared memory)
  kPhBigAsm = 1,    // big-front assembly (zero, scatter, extend-add)
  kPhBigPanel = 2,  // cluster panel factorization
  kPhBigUpd = 3,    // tiled trailing update
  kPhFwd = 4,       // forward solve
  kPhBwd = 5,       // backward solve
  kPhCluster = 6,   // fronts factored on chip in a cluster's shared memory
  kPhN = 7
};

// CUDA-event timing of kernel classes on the launching stream, plus a count
// of kernels launched. Events are recorded only while `on`.
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  double ms[kPhN] = {};
  long long launches[kPhN] = {};
  long long total_launches = 0;
  cudaEvent_t cur = nullptr;

  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(cudaStream_t st) {
    if (!on) return;
    cur = next();
    cudaEventRecord(cur, st);
  }
  void end(int phase, cudaStream_t st, int nlaunch) {
    total_launches += nlaunch;
    launches[phase] += nlaunch;
    if (!on) return;
    cudaEvent_t e = next();
    cudaEventRecord(e, st);
    marks.push_back({phase, {cur, e}});
  }
  // after the stream has been synchronized
  void collect() {
    for (auto& m : marks) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, m.second.first, m.second.second) == cudaSuccess)
        ms[m.first] += t;
    }
    marks.clear();
    used = 0;
  }
  void reset() {
    for (int i = 0; i < kPhN; i++) {
      ms[i] = 0.0;
      launches[i] = 0;
    }
    marks.clear();
    used = 0;
  }
  ~Prof() {
    for (auto e : pool) cudaEventDestroy(e);
  }
};

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
  int app;      // 1: blocked panels with a-posteriori threshold tests (big_app.cu)
  int pending;  // a-posteriori panels: candidate position to delay after the update, or -1
  long long ioff;  // front variables (fv[f], orig[f]) in the int pool
  long long doff;  // the front F (f x f, column-major) in the double pool
  long long woff;  // the panel's W columns (f x kBigPanelMax) in the double pool
  long long xoff;  // a-posteriori panels: the diagonal block's factor and tests
  double flops;
};

constexpr int kBigPanelMax = 32;
// doubles of per-front scratch for the a-posteriori panels (big_app.cu)
constexpr int kAppScratch = 1536;
// its first kBigPanelMax doubles: the largest magnitude in each of the next
// panel's columns over the rows below its block, left there (as the bits of
// non-negative doubles) by the trailing update of the previous panel
constexpr int kAppNextColmax = 0;
// ints of big-front level metadata (factor.cu fills, the host reads back)
constexpr int kBigMeta = 24;

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
  int* err;         // [4]: [0] failure bits (1: a pool ran out, 2: a front
                    // above its launch's on-chip size, 4: a big front in a
                    // level not prepared for one), [1] node of first error,
                    // [2] completion ticket of the trailing-update launch
  int* inertia;     // [2] pos, neg
  double* flops;    // [kWork] executed flops: [0] all fronts, [1] big panels,
                    // (a-posteriori panels: [5] panels, [6] pivots rejected by
                    // the a-posteriori tests, [7] candidates delayed in the
                    // diagonal block)
                    // [2] big trailing updates, [3] trailing-update bytes
                    // moved, [4] fronts factored on chip in a cluster
  BigFront* big;    // [nn] big fronts of the current level
  int* big_meta;    // [kBigMeta]: count, max f, max fs, count large, max fs
                    // large, class counts [5..9], class max f [10..14], max f
                    // large [15], a-posteriori fronts: count [16], max f [17],
                    // max fs [18], roots left with candidates: count [19], most
                    // candidates left [20], step counters and failure flag [21..23]
  int* class_list;  // [8][nn] big-front indices per size class (6: a-posteriori,
                    // 7: a-posteriori roots that finish with chained panels)
  int cf_limit[5];  // largest front of each on-chip class
  // fronts re-planned from a pivot record: partner[v] = the variable that
  // formed a 2x2 pivot with v in the record, -1 otherwise (nullptr without a
  // record)
  const int* partner;
  // factorization from element Hessian blocks (b200ldl_factor_elements): the
  // CSR value of entry e is the sum, from zero in order, of
  // asm_blocks[asm_src[q]] for q in [asm_ptr[e], asm_ptr[e + 1]); nullptr
  // when the factorization reads CSR values
  const long long* asm_ptr;
  const long long* asm_src;
  const double* asm_blocks;
};

// The CSR value of entry e: from the values, or assembled from the element
// blocks in the order of the assembly kernel (assembly.cu), so that a front
// receives the same bits either way.
__device__ __forceinline__ double csr_value(const DevState& s, const double* __restrict__ vals,
                                            long long e) {
  if (!s.asm_blocks) return vals[e];
  double v = 0.0;
  const long long q1 = s.asm_ptr[e + 1];
  for (long long q = s.asm_ptr[e]; q < q1; q++) v += s.asm_blocks[s.asm_src[q]];
  return v;
}

struct FactorParams {
  double ustab;
  double pivot_tol;
  int cholesky;
  // fronts above the shared-memory limit that have contribution rows are
  // factored in blocked panels with a-posteriori threshold tests
  // (big_app.cu) instead of the candidate-by-candidate search, from fronts
  // of app_min_f rows up
  int app;
  int app_min_f;
  // mixed precision: the contribution-block tiles of the a-posteriori panels'
  // trailing updates on the tensor cores (3xTF32, FP32 accumulation)
  int mixed;
};

// Largest front factored entirely in shared memory (fp64, ld = f | 1).
constexpr int kSmemFrontMax = 144;
constexpr int kFactorThreads = 256;

// fmax: the largest front the launch may meet on chip (its shared memory is
// sized for it); fronts above kSmemFrontMax go to the big-front path, which
// the host prepares for the level only with allow_big (else such a front
// stops the factorization with failure bit 4)
void launch_factor_level(const DevPlan& p, const DevState& s,
                         const int* level_nodes, int count, int fmax, int allow_big,
                         const FactorParams& prm, cudaStream_t stream,
                         const double* vals, const double* diag);
cudaError_t configure_factor_kernels();
size_t factor_smem_bytes(int f);

// Big-front pipeline for one level (see big.cu).
struct BigLevelInfo {
  int count, max_f, max_fs;
  int count_large, max_fs_large;
  int class_count[5], class_maxf[5];
  int cluster_launches;
  int max_f_large;  // largest front of class 5
  int count_app, max_f_app, max_fs_app;  // class 6: a-posteriori panels
};

// Fronts above kSmemFrontMax are factored on chip by a cluster of 1, 2, 4,
// 8 or 16 CTAs (class 0..4) when they fit in its distributed shared memory
// (cluster_front_limit(class)); larger ones (class 5) panel by panel from
// global memory.
int cluster_front_limit(int cl_index);
cudaError_t configure_cluster_front_kernels();
cudaError_t launch_cluster_fronts(const DevPlan& p, const DevState& s, const int* counts,
                                  const int* maxf, const double* vals, const double* diag,
                                  const FactorParams& prm, cudaStream_t stream, int nn);
// Class-5 fronts whose panel state fits one cluster's shared memory use the
// chained panel kernel (big_chain.cu); larger ones the single-candidate one.
// Panel width (32 or 16) the chained kernel uses for fronts up to f, 0 if
// its panel state does not fit.
int big_chain_panel_width(int f);
cudaError_t configure_big_chain_kernel();
cudaError_t launch_big_chain_panel(const DevState& s, const FactorParams& prm, int count,
                                   int max_f, int nb, const int* list, cudaStream_t stream);

// A-posteriori blocked panels (big_app.cu): every panel step of the class-6
// fronts in `list` (count of them, the largest with max_fs candidates) in
// one cooperative launch. counters: 3 zeroed ints in device memory;
// counters[2] is set if the step cap was reached (it is not when every step
// makes progress).
// `done` receives the roots whose panels left candidates (count in
// meta[19], most candidates left in meta[20]); meta[21..22] are the step
// counters and meta[23] the failure flag.
cudaError_t launch_app_level(const DevState& s, const FactorParams& prm, int count, int max_fs,
                             const int* list, int* done, int* meta, cudaStream_t stream);
cudaError_t configure_app_kernels();

cudaError_t launch_big_level(const DevPlan& p, const DevState& s, const BigLevelInfo& info,
                             const FactorParams& prm, const double* vals,
                             const double* diag, cudaStream_t stream, Prof& prof);
cudaError_t configure_big_kernels();

constexpr int kSolveThreads = 256;
// Right-hand sides per solve launch for a level whose largest front is fmax
// (0 if even one does not fit in shared memory).
int solve_rhs_chunk(int fmax, int nrhs);

int launch_forward_level(const DevPlan& p, const DevState& s,
                         const int* level_nodes, int count, double* x,
                         int ldx, int nrhs, double* upool, int fmax,
                         cudaStream_t stream);
int launch_backward_level(const DevPlan& p, const DevState& s,
                          const int* level_nodes, int count, double* x,
                          int ldx, int nrhs, int fmax, cudaStream_t stream);
cudaError_t configure_solve_kernels();

// Supernodes with fronts of at least kSolveBigFront rows are solved by a
// 16-CTA cluster each (solve_big.cu) when their vectors fit its shared memory.
constexpr int kSolveBigFront = 1024;
bool solve_big_fits(int f);
cudaError_t configure_solve_big_kernels();
int launch_forward_big(const DevPlan& p, const DevState& s, const int* nodes, int count,
                       double* x, int ldx, int nrhs, double* upool, int fmax,
                       cudaStream_t stream, cudaError_t* err);
int launch_backward_big(const DevPlan& p, const DevState& s, const int* nodes, int count,
                        double* x, int ldx, int nrhs, int fmax, cudaStream_t stream,
                        cudaError_t* err);

// per-system inertia of a batch of independent systems (batch.cu)
void launch_system_inertia(const DevState& s, const int* node_sys, int nn, int* sys_inertia,
                           cudaStream_t st);

// residuals and refinement helpers (refine.cu)
int refine_max_rhs();
void launch_value_gradient(int n, const int* rowp, const int* cols, const double* lam, int ldl,
                           const double* x, int ldx, int nr, double* gvals, double* gdiag,
                           cudaStream_t st);
void launch_residual(int n, const int* rowp, const int* cols, const double* vals,
                     const double* diag, const double* x, int ldx, const double* b, int ldb,
                     double* r, int ldr, int nr, cudaStream_t st);
void launch_colmax(int n, const double* v, int ld, int nr, double* out, cudaStream_t st);
void launch_infnorm(int n, const int* rowp, const int* cols, const double* vals,
                    const double* diag, double* out, cudaStream_t st);
void launch_axpy(int n, int nr, const double* d, int ldd, double* x, int ldx, cudaStream_t st);
void launch_copy_cols(int n, int nr, const double* src, int lds, double* dst, int ldd,
                      cudaStream_t st);
// the diagonal of one inertia-correction attempt; cls bit 0 = primal row
// (+dx), bit 1 = constraint row (-dc)
void launch_perturb_diag(int n, const double* diag, const unsigned char* cls, double dx,
                         double dc, double* out, cudaStream_t st);

// The device copy of an assembly plan (assembly.cu): its pattern's size and
// the per-CSR-entry contribution lists. Returns 0, or -1 without a plan.
int assembly_device_plan(const ::b200ldl_assembly* a, int* n, int* nnz, const long long** ptr,
                         const long long** src);

}  // namespace b200ldl
