// C-ABI of the B200 multifrontal LDL^T (declared in include/b200ldl.h).
//
// A handle owns: the host symbolic analysis, the device plan (assembly and
// extend-add maps, level lists), and the device pools of the last
// factorization. Errors are returned as status codes with a message kept on
// the handle; nothing aborts.
#include <cmath>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/b200ldl.h"
#include "ldl_internal.h"
#include "symbolic.h"

using namespace b200ldl;

namespace {

template <typename T>
struct DevBuf {
  T* ptr = nullptr;
  size_t count = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    count = 0;
  }
  cudaError_t alloc(size_t n) {
    release();
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&ptr, n * sizeof(T));
    if (e == cudaSuccess) count = n;
    else ptr = nullptr;
    return e;
  }
  cudaError_t upload(const std::vector<T>& h) {
    cudaError_t e = alloc(h.size());
    if (e != cudaSuccess) return e;
    if (!h.empty()) e = cudaMemcpy(ptr, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
  }
};

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const char* what)
      : std::runtime_error(std::string(what) + ": " + cudaGetErrorString(c)), code(c) {}
};

#define CK(call)                                        \
  do {                                                  \
    cudaError_t e__ = (call);                           \
    if (e__ != cudaSuccess) throw CudaError(e__, #call); \
  } while (0)

}  // namespace

struct b200ldl_handle {
  int n = 0, nnz = 0;
  int solver_type = B200LDL_LDL;
  double ustab = 0.01, pivot_tol = 1e-14, delay_growth = 2.0;
  int order = B200LDL_ORDER_NATURAL;
  cudaStream_t stream = nullptr;
  std::string last_error;

  // sym: the supernodal structure the factorization runs on; sym_ref: the
  // reference's symbolic structure (the same until a pivot order is reused)
  Symbolic sym, sym_ref;
  bool replanned = false;
  // 2x2 partners of the pivot record the structure was re-planned from
  std::vector<int> partner;
  DevBuf<int> d_partner;
  // precision of the big fronts' contribution-block updates; in MIXED mode
  // every solve is refined in FP64 against the matrix of the last factor
  int precision = B200LDL_FP64;
  int refine_max = 5;
  double refine_tol = 1e-12;
  bool factored_mixed = false;
  const double* last_vals = nullptr;
  // element-block source of the factorization in progress (nullptr: CSR
  // values)
  const long long* asm_ptr = nullptr;
  const long long* asm_src = nullptr;
  const double* asm_blocks = nullptr;
  const double* last_diag = nullptr;
  int last_iters = 0;
  double last_berr = 0.0;
  // inertia of the last FP64 factorization (-1: none yet), against which a
  // mixed factorization is checked, and the FP64 redos the checks caused
  int fp64_inertia[2] = {-1, -1};
  int mixed_fallbacks = 0;
  DevBuf<double> d_rhs_tmp;
  bool uploaded = false;
  // independent systems factored as one forest (1 for a single system)
  int nsys = 1;
  std::vector<int> node_sys;     // [num_nodes] system of each supernode
  std::vector<int> sys_inertia;  // [2 nsys] after a factorization
  DevBuf<int> d_node_sys, d_sys_inertia;
  std::vector<int> h_rowp, h_cols;  // the pattern, for residuals
  DevBuf<int> d_rowp, d_cols;
  DevBuf<double> d_refine, d_norms;
  // host copies of the plan (uploaded lazily on the first factorization so
  // that the symbolic phase runs on machines without a GPU)
  std::vector<int> hp_ns, hp_nc, hp_kid_ptr, hp_kids, hp_cmap, hp_scat_csr, hp_scat_row,
      hp_scat_col, hp_level_nodes;
  std::vector<int64_t> hp_scat_ptr;
  int num_levels = 0;
  std::vector<int> level_ptr;  // host copy
  // a level whose fronts cannot exceed the shared-memory limit, whatever the
  // delays, needs no big-front launch (and no host read-back)
  std::vector<char> level_may_big;
  // per level: whether the host prepares big fronts (a device sync per such
  // level): the levels that had one in the last factorization, the levels
  // whose bound allows one until then
  std::vector<char> level_big;
  std::vector<int> level_fbound;  // per level: bound on its on-chip fronts (shared memory sizing)
  // per level: the on-chip front size its small-front launch is given, the
  // last factorization's largest front plus slack (the bound until then)
  std::vector<int> level_fcap;
  std::vector<int> h_ns, h_nc;

  // device plan
  DevBuf<int> d_ns, d_nc, d_var_ptr, d_node_to_var, d_cptr, d_contrib_rows, d_cmap,
      d_kid_ptr, d_kids, d_scat_csr, d_scat_row, d_scat_col, d_level_nodes;
  DevBuf<int64_t> d_scat_ptr;
  DevPlan plan{};

  // device state
  DevBuf<int> d_f, d_fs, d_npiv, d_ndel, d_L_ld, d_cb_ld, d_ivars, d_err, d_inertia;
  DevBuf<int64_t> d_fv_off, d_L_off, d_cb_off, d_u_off;
  DevBuf<double> d_dpool, d_flops, d_upool, d_vals, d_diag, d_x;
  DevBuf<unsigned long long> d_used;
  DevBuf<BigFront> d_big;
  DevBuf<int> d_big_meta;
  DevBuf<int> d_class_list;
  // inertia correction: per row, bit 0 = primal (+delta_x), bit 1 =
  // constraint (-delta_c); the perturbed diagonal of the last attempt
  DevBuf<unsigned char> d_pclass;
  DevBuf<double> d_pdiag;
  bool have_pclass = false;
  unsigned long long icap = 0, dcap = 0;
  DevState st{};

  // results of the last factorization
  bool factored = false;
  int inertia[2] = {0, 0};
  unsigned long long used[3] = {0, 0, 0};
  double exec_flops = 0.0;
  int fmax = 0;
  std::vector<int> level_fmax;
  // solve schedule of the last factorization: per level, the supernodes for
  // the one-CTA kernels then those for the cluster kernels
  std::vector<int> solve_ptr;    // [2 * levels + 1]
  std::vector<int> solve_nodes;  // host copy of d_solve_nodes
  std::vector<int> solve_fmax;   // [2 * levels]: largest front of each list
  DevBuf<int> d_solve_nodes;
  Prof prof;
  double flops4[kWork] = {};
  double sum_delayed = 0.0;
};

namespace {

int fail(b200ldl_t h, int code, const char* fmt, ...) {
  if (h) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    h->last_error = buf;
  }
  return code;
}

// Build the static assembly / extend-add maps and the level lists.
void build_plan(b200ldl_t h, const int* rowp, const int* cols) {
  const Symbolic& s = h->sym;
  const int n = s.n;
  const int nn = s.num_nodes;
  std::vector<int> ns(nn), nc(nn);
  for (int k = 0; k < nn; k++) {
    ns[k] = s.node_ptr[k + 1] - s.node_ptr[k];
    nc[k] = s.contrib_ptr[k + 1] - s.contrib_ptr[k];
  }
  std::vector<int> kid_ptr(s.children_ptr.begin(), s.children_ptr.begin() + nn + 1);
  std::vector<int> kids(s.children.begin(), s.children.begin() + kid_ptr[nn]);

  // positions of the front variables of node k (own vars then contrib rows)
  std::vector<int> where(n, -1);
  auto put = [&](int v, int pos) {
    if (v < 0 || v >= n) throw std::runtime_error("front variable out of range");
    if (pos >= 0 && where[v] >= 0) throw std::runtime_error("variable listed twice in one front");
    where[v] = pos;
  };
  auto mark = [&](int k, int sign) {
    for (int j = 0; j < ns[k]; j++) put(s.node_to_var[s.node_ptr[k] + j], sign ? j : -1);
    for (int t = 0; t < nc[k]; t++) put(s.contrib_rows[s.contrib_ptr[k] + t], sign ? ns[k] + t : -1);
  };

  std::vector<int> cmap(s.contrib_rows.size(), -1);
  std::vector<int64_t> scat_ptr(nn + 1, 0);
  std::vector<int> scat_csr, scat_row, scat_col;
  scat_csr.reserve(rowp[n]);
  scat_row.reserve(rowp[n]);
  scat_col.reserve(rowp[n]);
  const int* ip = s.iperm.data();
  for (int k = 0; k < nn; k++) {
    mark(k, 1);
    for (int j = 0; j < ns[k]; j++) {
      const int var = s.node_to_var[s.node_ptr[k] + j];
      const int pj = ip[var];
      for (int e = rowp[var]; e < rowp[var + 1]; e++) {
        const int i = cols[e];
        if (ip[i] < pj) continue;
        const int w = where[i];
        // an entry eliminated here must have its row in this front
        if (w < 0) throw std::runtime_error("matrix entry outside the front that eliminates it");
        scat_csr.push_back(e);
        scat_row.push_back(w);
        scat_col.push_back(j);
      }
    }
    scat_ptr[k + 1] = (int64_t)scat_csr.size();
    // children's contribution rows -> positions in this front
    for (int c = kid_ptr[k]; c < kid_ptr[k + 1]; c++) {
      const int ch = kids[c];
      for (int t = s.contrib_ptr[ch]; t < s.contrib_ptr[ch + 1]; t++) {
        const int w = where[s.contrib_rows[t]];
        if (w < 0) throw std::runtime_error("contribution row missing from the parent front");
        cmap[t] = w;
      }
    }
    mark(k, 0);
  }
  for (int k = 0; k < nn; k++) {
    if (s.parent[k] < 0 && nc[k] > 0)
      throw std::runtime_error("root supernode with contribution rows");
  }

  // levels: leaves 0, parent = 1 + max(children)
  std::vector<int> level(nn, 0);
  bool post = true;
  for (int k = 0; k < nn; k++)
    if (s.parent[k] >= 0 && s.parent[k] <= k) post = false;
  if (post) {
    for (int k = 0; k < nn; k++)
      if (s.parent[k] >= 0) level[s.parent[k]] = std::max(level[s.parent[k]], level[k] + 1);
  } else {
    bool changed = true;
    while (changed) {
      changed = false;
      for (int k = 0; k < nn; k++) {
        const int p = s.parent[k];
        if (p >= 0 && level[p] < level[k] + 1) {
          level[p] = level[k] + 1;
          changed = true;
        }
      }
    }
  }
  int nl = 0;
  for (int k = 0; k < nn; k++) nl = std::max(nl, level[k] + 1);
  if (nn == 0) nl = 0;
  std::vector<int> lptr(nl + 1, 0), lnodes(nn);
  for (int k = 0; k < nn; k++) lptr[level[k] + 1]++;
  for (int l = 0; l < nl; l++) lptr[l + 1] += lptr[l];
  {
    std::vector<int> fill(lptr.begin(), lptr.end());
    for (int k = 0; k < nn; k++) lnodes[fill[level[k]]++] = k;
  }
  h->num_levels = nl;
  h->level_ptr = lptr;
  // an upper bound on every front's run-time size: a child delays at most
  // all of its candidates, so fs <= ns + sum of the children's bounds
  {
    std::vector<long long> fsb(nn, 0);
    std::vector<int> order(nn);
    for (int k = 0; k < nn; k++) order[k] = k;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return level[a] < level[b]; });
    for (int k : order) {
      long long b = ns[k];
      for (int c = kid_ptr[k]; c < kid_ptr[k + 1]; c++) b += fsb[kids[c]];
      fsb[k] = b;
    }
    h->level_may_big.assign(nl, 0);
    h->level_fbound.assign(nl, 1);
    for (int k = 0; k < nn; k++) {
      const long long fb = fsb[k] + nc[k];
      if (fb > kSmemFrontMax) h->level_may_big[level[k]] = 1;
      // the on-chip front of the level's small-front launch: sized for its
      // largest bound, so that small fronts leave room for more CTAs per SM
      h->level_fbound[level[k]] =
          std::max(h->level_fbound[level[k]], (int)std::min<long long>(fb, kSmemFrontMax));
    }
    h->level_fcap = h->level_fbound;
    h->level_big = h->level_may_big;
  }
  h->h_ns = ns;
  h->h_nc = nc;
  h->hp_ns = std::move(ns);
  h->hp_nc = std::move(nc);
  h->hp_kid_ptr = std::move(kid_ptr);
  h->hp_kids = std::move(kids);
  h->hp_cmap = std::move(cmap);
  h->hp_scat_ptr = std::move(scat_ptr);
  h->hp_scat_csr = std::move(scat_csr);
  h->hp_scat_row = std::move(scat_row);
  h->hp_scat_col = std::move(scat_col);
  h->hp_level_nodes = std::move(lnodes);

  // pool estimates from the symbolic fronts, scaled by the delay growth; a
  // structure re-planned from a pivot record already holds its delays, and
  // its big fronts take the a-posteriori panels, which need no chained-panel
  // scratch except at roots (which may finish with chained panels)
  double ints = 0.0, dbl = 0.0;
  for (int k = 0; k < nn; k++) {
    const double f = h->h_ns[k] + h->h_nc[k];
    ints += 2.0 * f;
    dbl += f * h->h_ns[k] + (double)h->h_nc[k] * h->h_nc[k];
    if (f > kSmemFrontMax) dbl += f * f + (kBigPanelMax + 2.0) * f + kAppScratch;
    const bool chain = h->replanned ? (f > kSmemFrontMax && h->h_nc[k] == 0)
                                    : f > cluster_front_limit(4);
    if (chain) dbl += f * f + 32.0 * f;  // chained panels' scratch
  }
  const double g = h->replanned ? 1.0 : std::max(1.0, h->delay_growth);
  h->icap = (unsigned long long)(ints * g * 1.5) + (1u << 16);
  h->dcap = (unsigned long long)(dbl * g * 1.5) + (1u << 20);
}

// Supernodal structure from a pivot record: supernode k's pivot columns
// become the variables it eliminated, in the order it eliminated them (a 2x2
// pair stays adjacent), and the candidates it delayed join its contribution
// rows ahead of the rows it already had. The elimination tree and the node
// numbering are kept, so the permutation is the elimination order the record
// describes. rec_f/rec_npiv/rec_ndel: per supernode; rec_fv: each
// supernode's front variables after pivoting (f entries: pivots with 2x2
// pairs encoded -(v+1), delayed, contribution rows), one after another.
Symbolic replan_from_record(const Symbolic& tree, const int* rec_f, const int* rec_npiv,
                            const int* rec_ndel, const int* rec_fv, std::vector<int>& partner) {
  const int n = tree.n, nn = tree.num_nodes;
  Symbolic s;
  s.n = n;
  s.num_nodes = nn;
  s.permuted = true;
  s.children_ptr = tree.children_ptr;
  s.children = tree.children;
  s.parent = tree.parent;
  s.node_ptr.assign(1, 0);
  s.contrib_ptr.assign(1, 0);
  s.node_to_var.reserve(n);
  long long off = 0;
  for (int k = 0; k < nn; k++) {
    const int f = rec_f[k], np = rec_npiv[k], nd = rec_ndel[k];
    if (f < 0 || np < 0 || nd < 0 || np + nd > f)
      throw std::invalid_argument("pivot record: inconsistent front sizes");
    const int* fv = rec_fv + off;
    for (int t = 0; t < np; t++) {
      const int v = fv[t] >= 0 ? fv[t] : -fv[t] - 1;
      s.node_to_var.push_back(v);
    }
    // 2x2 pivots are consecutive pairs of encoded entries
    for (int t = 0; t < np;) {
      if (fv[t] < 0 && t + 1 < np && fv[t + 1] < 0) {
        const int a = -fv[t] - 1, b = -fv[t + 1] - 1;
        if (a >= 0 && a < n && b >= 0 && b < n) {
          partner[a] = b;
          partner[b] = a;
        }
        t += 2;
      } else {
        t += 1;
      }
    }
    for (int t = np; t < f; t++) s.contrib_rows.push_back(fv[t]);
    s.node_ptr.push_back((int)s.node_to_var.size());
    s.contrib_ptr.push_back((int)s.contrib_rows.size());
    off += f;
  }
  if ((int)s.node_to_var.size() != n)
    throw std::invalid_argument("pivot record: pivots do not cover every variable once");
  s.iperm.assign(n, -1);
  for (int q = 0; q < n; q++) {
    const int v = s.node_to_var[q];
    if (v < 0 || v >= n || s.iperm[v] >= 0)
      throw std::invalid_argument("pivot record: pivots do not cover every variable once");
    s.iperm[v] = q;
  }
  s.perm = s.node_to_var;
  return s;
}

// Switch the handle to structure `s` (the device plan is rebuilt at the next
// factorization; the last factor is dropped).
void use_structure(b200ldl_t h, Symbolic&& s) {
  Symbolic old = std::move(h->sym);
  h->sym = std::move(s);
  try {
    build_plan(h, h->h_rowp.data(), h->h_cols.data());
  } catch (...) {
    h->sym = std::move(old);
    build_plan(h, h->h_rowp.data(), h->h_cols.data());
    throw;
  }
  h->uploaded = false;
  h->factored = false;
  h->fmax = 0;
}

void upload_plan(b200ldl_t h) {
  if (h->uploaded) return;
  const Symbolic& s = h->sym;
  const int nn = s.num_nodes;
  CK(h->d_ns.upload(h->hp_ns));
  CK(h->d_nc.upload(h->hp_nc));
  CK(h->d_var_ptr.upload(s.node_ptr));
  CK(h->d_node_to_var.upload(s.node_to_var));
  CK(h->d_cptr.upload(s.contrib_ptr));
  CK(h->d_contrib_rows.upload(s.contrib_rows));
  CK(h->d_cmap.upload(h->hp_cmap));
  CK(h->d_kid_ptr.upload(h->hp_kid_ptr));
  CK(h->d_kids.upload(h->hp_kids));
  CK(h->d_scat_ptr.upload(h->hp_scat_ptr));
  CK(h->d_scat_csr.upload(h->hp_scat_csr));
  CK(h->d_scat_row.upload(h->hp_scat_row));
  CK(h->d_scat_col.upload(h->hp_scat_col));
  CK(h->d_level_nodes.upload(h->hp_level_nodes));
  CK(h->d_rowp.upload(h->h_rowp));
  CK(h->d_cols.upload(h->h_cols));
  if (h->replanned) CK(h->d_partner.upload(h->partner));

  DevPlan& p = h->plan;
  p.n = s.n;
  p.num_nodes = nn;
  p.ns = h->d_ns.ptr;
  p.nc = h->d_nc.ptr;
  p.var_ptr = h->d_var_ptr.ptr;
  p.node_to_var = h->d_node_to_var.ptr;
  p.cptr = h->d_cptr.ptr;
  p.contrib_rows = h->d_contrib_rows.ptr;
  p.cmap = h->d_cmap.ptr;
  p.kid_ptr = h->d_kid_ptr.ptr;
  p.kids = h->d_kids.ptr;
  p.scat_ptr = h->d_scat_ptr.ptr;
  p.scat_csr = h->d_scat_csr.ptr;
  p.scat_row = h->d_scat_row.ptr;
  p.scat_col = h->d_scat_col.ptr;

  // per-node state
  CK(h->d_f.alloc(nn));
  CK(h->d_fs.alloc(nn));
  CK(h->d_npiv.alloc(nn));
  CK(h->d_ndel.alloc(nn));
  CK(h->d_L_ld.alloc(nn));
  CK(h->d_cb_ld.alloc(nn));
  CK(h->d_fv_off.alloc(nn));
  CK(h->d_L_off.alloc(nn));
  CK(h->d_cb_off.alloc(nn));
  CK(h->d_u_off.alloc(nn));
  CK(h->d_err.alloc(4));
  CK(h->d_inertia.alloc(2));
  CK(h->d_flops.alloc(kWork));
  CK(h->d_used.alloc(3));
  CK(h->d_big.alloc(nn));
  CK(h->d_big_meta.alloc(kBigMeta));
  CK(h->d_class_list.alloc((size_t)8 * std::max(1, nn)));
  h->uploaded = true;
}

void bind_state(b200ldl_t h) {
  DevState& st = h->st;
  st.f = h->d_f.ptr;
  st.fs = h->d_fs.ptr;
  st.npiv = h->d_npiv.ptr;
  st.ndel = h->d_ndel.ptr;
  st.fv_off = h->d_fv_off.ptr;
  st.L_off = h->d_L_off.ptr;
  st.L_ld = h->d_L_ld.ptr;
  st.cb_off = h->d_cb_off.ptr;
  st.cb_ld = h->d_cb_ld.ptr;
  st.u_off = h->d_u_off.ptr;
  st.ivars = h->d_ivars.ptr;
  st.dpool = h->d_dpool.ptr;
  st.used = h->d_used.ptr;
  st.icap = h->icap;
  st.dcap = h->dcap;
  st.err = h->d_err.ptr;
  st.inertia = h->d_inertia.ptr;
  st.flops = h->d_flops.ptr;
  st.big = h->d_big.ptr;
  st.big_meta = h->d_big_meta.ptr;
  st.class_list = h->d_class_list.ptr;
  for (int c = 0; c < 5; c++) st.cf_limit[c] = cluster_front_limit(c);
  st.partner = h->replanned ? h->d_partner.ptr : nullptr;
  st.asm_ptr = h->asm_ptr;
  st.asm_src = h->asm_src;
  st.asm_blocks = h->asm_blocks;
}

void ensure_pools(b200ldl_t h) {
  upload_plan(h);
  if (h->d_ivars.count < h->icap) CK(h->d_ivars.alloc(h->icap));
  if (h->d_dpool.count < h->dcap) CK(h->d_dpool.alloc(h->dcap));
  bind_state(h);
}

// Kernel attributes (shared memory sizes, cluster sizes) are set once per
// device, on the device that is current, under a lock so that threads
// driving different devices or handles do not race.
void configure_device_kernels() {
  static std::mutex mu;
  static std::vector<char> done;
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if ((int)done.size() > dev && done[dev]) return;
  CK(configure_factor_kernels());
  CK(configure_solve_kernels());
  CK(configure_solve_big_kernels());
  CK(configure_big_kernels());
  CK(configure_app_kernels());
  if ((int)done.size() <= dev) done.resize(dev + 1, 0);
  done[dev] = 1;
}

void level_fronts(b200ldl_t h);

void run_factor_once(b200ldl_t h, const double* vals, const double* diag, bool mixed) {
  configure_device_kernels();
  // fronts re-planned from a pivot record are expected to accept their
  // candidates where they stand: their big fronts take the blocked panels
  // with a-posteriori tests
  FactorParams prm{h->ustab, h->pivot_tol, h->solver_type == B200LDL_CHOLESKY ? 1 : 0,
                   (h->replanned && h->solver_type != B200LDL_CHOLESKY) ? 1 : 0, 0, 0};
  prm.mixed = (prm.app && mixed) ? 1 : 0;
  h->factored_mixed = prm.mixed != 0;
  h->last_vals = vals;
  h->last_diag = diag;
  for (int attempt = 0; attempt < 12; attempt++) {
    ensure_pools(h);
    CK(cudaMemsetAsync(h->d_used.ptr, 0, 3 * sizeof(unsigned long long), h->stream));
    CK(cudaMemsetAsync(h->d_err.ptr, 0, sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_err.ptr + 1, 0xff, sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_err.ptr + 2, 0, 2 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_inertia.ptr, 0, 2 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_flops.ptr, 0, kWork * sizeof(double), h->stream));
    CK(cudaMemsetAsync(h->d_ndel.ptr, 0, sizeof(int) * std::max(1, h->sym.num_nodes), h->stream));
    for (int l = 0; l < h->num_levels; l++) {
      const int b = h->level_ptr[l];
      const int cnt = h->level_ptr[l + 1] - b;
      if (h->level_big[l])
        CK(cudaMemsetAsync(h->d_big_meta.ptr, 0, kBigMeta * sizeof(int), h->stream));
      h->prof.begin(h->stream);
      launch_factor_level(h->plan, h->st, h->d_level_nodes.ptr + b, cnt, h->level_fcap[l],
                          h->level_big[l], prm, h->stream, vals, diag);
      h->prof.end(kPhFront, h->stream, 1);
      CK(cudaGetLastError());
      if (!h->level_big[l]) continue;
      int meta[kBigMeta];
      CK(cudaMemcpyAsync(meta, h->d_big_meta.ptr, kBigMeta * sizeof(int), cudaMemcpyDeviceToHost,
                         h->stream));
      CK(cudaStreamSynchronize(h->stream));
      if (meta[0] > 0) {
        BigLevelInfo info{};
        info.count = meta[0];
        info.max_f = meta[1];
        info.max_fs = meta[2];
        info.count_large = meta[3];
        info.max_fs_large = meta[4];
        info.max_f_large = meta[15];
        info.count_app = meta[16];
        info.max_f_app = meta[17];
        info.max_fs_app = meta[18];
        info.cluster_launches = 0;
        for (int c = 0; c < 5; c++) {
          info.class_count[c] = meta[5 + c];
          info.class_maxf[c] = meta[10 + c];
          if (meta[5 + c] > 0) info.cluster_launches++;
        }
        CK(launch_big_level(h->plan, h->st, info, prm, vals, diag,
                            h->stream, h->prof));
      }
    }
    CK(cudaGetLastError());
    int err[2];
    CK(cudaMemcpyAsync(err, h->d_err.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->used, h->d_used.ptr, 3 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToHost, h->stream));
    CK(cudaMemcpyAsync(h->inertia, h->d_inertia.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaMemcpyAsync(h->flops4, h->d_flops.ptr, kWork * sizeof(double),
                       cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->exec_flops = h->flops4[0];
    h->prof.collect();
    if (err[0] == 0) {
      if (h->nsys > 1 && h->solver_type != B200LDL_CHOLESKY) {
        if (h->d_node_sys.count < h->node_sys.size()) CK(h->d_node_sys.upload(h->node_sys));
        if (h->d_sys_inertia.count < (size_t)2 * h->nsys) CK(h->d_sys_inertia.alloc(2 * h->nsys));
        CK(cudaMemsetAsync(h->d_sys_inertia.ptr, 0, 2 * h->nsys * sizeof(int), h->stream));
        launch_system_inertia(h->st, h->d_node_sys.ptr, h->sym.num_nodes, h->d_sys_inertia.ptr,
                              h->stream);
        CK(cudaGetLastError());
        h->sys_inertia.assign(2 * h->nsys, 0);
        CK(cudaMemcpyAsync(h->sys_inertia.data(), h->d_sys_inertia.ptr,
                           2 * h->nsys * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
      }
      h->factored = true;
      // on-chip sizes for the next factorization: this one's largest front
      // per level, with room for a quarter more (at least 8 rows) of delays
      level_fronts(h);
      for (int l = 0; l < h->num_levels; l++) {
        const int fm = h->level_fmax[l];
        h->level_fcap[l] = std::min(h->level_fbound[l],
                                    std::min(kSmemFrontMax, fm + std::max(8, fm / 4)));
        h->level_big[l] = fm > kSmemFrontMax ? 1 : 0;
      }
      return;
    }
    if (err[0] & 4) {
      // a front went big in a level not prepared for one: every level whose
      // bound allows one is prepared
      h->level_big = h->level_may_big;
    }
    if (err[0] & 2) {
      // a front outgrew its launch's on-chip size: every level gets its
      // bound, which no front can exceed
      h->level_fcap = h->level_fbound;
    }
    if (err[0] & 1) {
      // a pool ran out: grow both (the counters stop being meaningful after
      // the first failure, so grow geometrically) and factor again
      h->icap = std::max<unsigned long long>(h->icap * 2, h->used[0] + (1u << 16));
      h->dcap = std::max<unsigned long long>(h->dcap * 2, h->used[1] + (1u << 20));
    }
  }
  throw std::runtime_error("factor storage did not converge after repeated growth");
}

// A mixed-precision factorization is kept only if its inertia equals that of
// the last FP64 factorization of the pattern (the one whose pivot record the
// handle reuses, or a later one); otherwise, and whenever no FP64 inertia is
// known yet, the factorization runs in FP64. Rounding at FP32 level in the
// contribution blocks can flip the sign of a pivot that cancellation makes
// tiny, so the FP64 factorization decides the inertia in that case.
void run_factor(b200ldl_t h, const double* vals, const double* diag) {
  const bool mixed = h->replanned && h->precision == B200LDL_MIXED &&
                     h->solver_type != B200LDL_CHOLESKY && h->fp64_inertia[0] >= 0;
  if (mixed) {
    run_factor_once(h, vals, diag, true);
    if (!h->factored_mixed || (h->inertia[0] == h->fp64_inertia[0] &&
                               h->inertia[1] == h->fp64_inertia[1]))
      return;
    h->mixed_fallbacks++;
  }
  run_factor_once(h, vals, diag, false);
  h->fp64_inertia[0] = h->inertia[0];
  h->fp64_inertia[1] = h->inertia[1];
}


// largest front of every level of the last factorization
void level_fronts(b200ldl_t h) {
  const int nn = h->sym.num_nodes;
  std::vector<int> f(nn);
  CK(cudaMemcpy(f.data(), h->d_f.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
  h->level_fmax.assign(h->num_levels, 1);
  h->solve_ptr.assign(2 * h->num_levels + 1, 0);
  h->solve_fmax.assign(2 * h->num_levels, 1);
  h->solve_nodes.clear();
  int m = 1;
  for (int l = 0; l < h->num_levels; l++) {
    for (int pass = 0; pass < 2; pass++) {
      h->solve_ptr[2 * l + pass] = (int)h->solve_nodes.size();
      for (int q = h->level_ptr[l]; q < h->level_ptr[l + 1]; q++) {
        const int node = h->hp_level_nodes[q];
        const int fn = f[node];
        const bool big = fn >= kSolveBigFront && solve_big_fits(fn);
        if (big != (pass == 1)) continue;
        h->solve_nodes.push_back(node);
        h->solve_fmax[2 * l + pass] = std::max(h->solve_fmax[2 * l + pass], fn);
        if (!big) m = std::max(m, fn);
      }
    }
    for (int q = h->level_ptr[l]; q < h->level_ptr[l + 1]; q++)
      h->level_fmax[l] = std::max(h->level_fmax[l], f[h->hp_level_nodes[q]]);
  }
  h->solve_ptr[2 * h->num_levels] = (int)h->solve_nodes.size();
  if (h->d_solve_nodes.count < h->solve_nodes.size())
    CK(h->d_solve_nodes.alloc(h->solve_nodes.size()));
  if (!h->solve_nodes.empty())
    CK(cudaMemcpy(h->d_solve_nodes.ptr, h->solve_nodes.data(),
                  h->solve_nodes.size() * sizeof(int), cudaMemcpyHostToDevice));
  h->fmax = m;  // largest front left to the one-CTA kernels
}

void run_solve(b200ldl_t h, int nrhs, double* x, int ldx) {
  if (h->fmax == 0) level_fronts(h);
  if (solve_rhs_chunk(h->fmax, 1) < 1)
    throw std::runtime_error("front too large for the solve kernels");
  const size_t need = (size_t)h->used[2] * nrhs;
  if (h->d_upool.count < need) CK(h->d_upool.alloc(need));
  const int* nodes = h->d_solve_nodes.ptr;
  cudaError_t err = cudaSuccess;
  for (int l = 0; l < h->num_levels; l++) {
    const int s0 = h->solve_ptr[2 * l], s1 = h->solve_ptr[2 * l + 1];
    const int s2 = h->solve_ptr[2 * l + 2];
    h->prof.begin(h->stream);
    int nl = launch_forward_level(h->plan, h->st, nodes + s0, s1 - s0, x, ldx, nrhs,
                                  h->d_upool.ptr, h->solve_fmax[2 * l], h->stream);
    nl += launch_forward_big(h->plan, h->st, nodes + s1, s2 - s1, x, ldx, nrhs, h->d_upool.ptr,
                             h->solve_fmax[2 * l + 1], h->stream, &err);
    CK(err);
    h->prof.end(kPhFwd, h->stream, nl);
  }
  for (int l = h->num_levels - 1; l >= 0; l--) {
    const int s0 = h->solve_ptr[2 * l], s1 = h->solve_ptr[2 * l + 1];
    const int s2 = h->solve_ptr[2 * l + 2];
    h->prof.begin(h->stream);
    int nl = launch_backward_level(h->plan, h->st, nodes + s0, s1 - s0, x, ldx, nrhs,
                                   h->solve_fmax[2 * l], h->stream);
    nl += launch_backward_big(h->plan, h->st, nodes + s1, s2 - s1, x, ldx, nrhs,
                              h->solve_fmax[2 * l + 1], h->stream, &err);
    CK(err);
    h->prof.end(kPhBwd, h->stream, nl);
  }
  CK(cudaGetLastError());
}

template <typename F>
int guarded(b200ldl_t h, F&& fn) {
  if (!h) return -1;
  try {
    h->last_error.clear();
    return fn();
  } catch (const CudaError& e) {
    cudaGetLastError();
    return fail(h, -3, "%s", e.what());
  } catch (const std::bad_alloc&) {
    return fail(h, -2, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(h, -4, "%s", e.what());
  }
}

// x = K^-1 b with FP64 iterative refinement against the CSR values `vals`
// and `diag` (device), every column until its backward error is <= tol or
// max_iter corrections were made; berr_out (host, nrhs entries) may be null.
void refine_impl(b200ldl_t h, const double* vals, const double* diag, int nrhs, const double* b,
                 int ldb, double* x, int ldx, int max_iter, double tol, double* berr_out,
                 int* iters_out) {
    if (iters_out) *iters_out = 0;
    if (nrhs == 0 || h->n == 0) return;
    const int n = h->n;
    const int chunk = refine_max_rhs();
    if (h->d_refine.count < (size_t)n * chunk) CK(h->d_refine.alloc((size_t)n * chunk));
    if (h->d_norms.count < (size_t)(1 + 3 * chunk)) CK(h->d_norms.alloc(1 + 3 * chunk));
    double* r = h->d_refine.ptr;
    double* nrm = h->d_norms.ptr;  // [0] ||K||, [1..] ||b||, ||x||, ||r|| per column
    CK(cudaMemsetAsync(nrm, 0, sizeof(double), h->stream));
    launch_infnorm(n, h->d_rowp.ptr, h->d_cols.ptr, vals, diag, nrm, h->stream);
    int max_it_done = 0;
    double worst = 0.0;
    for (int c0 = 0; c0 < nrhs; c0 += chunk) {
      const int nr = std::min(chunk, nrhs - c0);
      const double* bc = b + (size_t)ldb * c0;
      double* xc = x + (size_t)ldx * c0;
      launch_copy_cols(n, nr, bc, ldb, xc, ldx, h->stream);
      run_solve(h, nr, xc, ldx);
      CK(cudaMemsetAsync(nrm + 1, 0, sizeof(double) * chunk, h->stream));
      launch_colmax(n, bc, ldb, nr, nrm + 1, h->stream);
      int it = 0;
      for (;; it++) {
        launch_residual(n, h->d_rowp.ptr, h->d_cols.ptr, vals, diag, xc, ldx, bc, ldb, r, n, nr,
                        h->stream);
        CK(cudaMemsetAsync(nrm + 1 + chunk, 0, sizeof(double) * 2 * chunk, h->stream));
        launch_colmax(n, xc, ldx, nr, nrm + 1 + chunk, h->stream);
        launch_colmax(n, r, n, nr, nrm + 1 + 2 * chunk, h->stream);
        double hn[1 + 3 * 8];
        CK(cudaMemcpyAsync(hn, nrm, sizeof(double) * (1 + 3 * chunk), cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        bool ok = true;
        for (int c = 0; c < nr; c++) {
          const double den = hn[0] * hn[1 + chunk + c] + hn[1 + c];
          const double be = den > 0.0 ? hn[1 + 2 * chunk + c] / den : 0.0;
          if (berr_out) berr_out[c0 + c] = be;
          worst = std::max(worst, be);
          if (!(be <= tol)) ok = false;
        }
        if (ok || it >= max_iter) break;
        run_solve(h, nr, r, n);
        launch_axpy(n, nr, r, n, xc, ldx, h->stream);
      }
      max_it_done = std::max(max_it_done, it);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    h->prof.collect();
    if (iters_out) *iters_out = max_it_done;
    h->last_iters = max_it_done;
    h->last_berr = worst;
}

}  // namespace

extern "C" {

int b200ldl_create(b200ldl_t* out, int n, int nnz, const int* rowp, const int* cols,
                   int solver_type, double ustab, double pivot_tol, double delay_growth,
                   int order) {
  if (!out) return -1;
  *out = nullptr;
  if (n < 0 || nnz < 0 || (n > 0 && (!rowp || !cols))) return -1;
  if (solver_type != B200LDL_LDL && solver_type != B200LDL_CHOLESKY) return -1;
  if (order < 0 || order > B200LDL_ORDER_GRAPH_ND || order == B200LDL_ORDER_MULTI_COLOR)
    return -1;
  if (n > 0 && (rowp[0] != 0 || rowp[n] != nnz)) return -1;
  for (int i = 0; i < n; i++)
    if (rowp[i + 1] < rowp[i]) return -1;
  for (int e = 0; e < nnz; e++)
    if (cols[e] < 0 || cols[e] >= n) return -1;
  auto h = std::make_unique<b200ldl_handle>();
  h->n = n;
  h->nnz = nnz;
  h->solver_type = solver_type;
  h->ustab = ustab;
  h->pivot_tol = pivot_tol;
  h->delay_growth = delay_growth;
  h->order = order;
  int st = guarded(h.get(), [&]() {
    h->sym = analyze(static_cast<Ordering>(order), n, rowp, cols);
    build_plan(h.get(), rowp, cols);
    h->h_rowp.assign(rowp, rowp + n + 1);
    h->h_cols.assign(cols, cols + nnz);
    return 0;
  });
  if (st != 0) {
    std::fprintf(stderr, "b200ldl_create: %s\n", h->last_error.c_str());
    return st;
  }
  *out = h.release();
  return 0;
}

int b200ldl_create_batch(b200ldl_t* out, int nsys, const int* sys_n, const int* sys_nnz,
                         const int* rowp_cat, const int* cols_cat, int solver_type,
                         double ustab, double pivot_tol, double delay_growth, int order) {
  if (!out) return -1;
  *out = nullptr;
  if (nsys < 1 || !sys_n || !sys_nnz || !rowp_cat || !cols_cat) return -1;
  if (solver_type != B200LDL_LDL && solver_type != B200LDL_CHOLESKY) return -1;
  if (order < 0 || order > B200LDL_ORDER_GRAPH_ND || order == B200LDL_ORDER_MULTI_COLOR)
    return -1;
  // validate every system and build the block-diagonal pattern
  long long ntot = 0, nztot = 0;
  {
    long long ro = 0, co = 0;
    for (int si = 0; si < nsys; si++) {
      const int n = sys_n[si], nnz = sys_nnz[si];
      if (n < 0 || nnz < 0) return -1;
      const int* rowp = rowp_cat + ro;
      const int* cols = cols_cat + co;
      if (rowp[0] != 0 || rowp[n] != nnz) return -1;
      for (int i = 0; i < n; i++)
        if (rowp[i + 1] < rowp[i]) return -1;
      for (int e = 0; e < nnz; e++)
        if (cols[e] < 0 || cols[e] >= n) return -1;
      ro += n + 1;
      co += nnz;
      ntot += n;
      nztot += nnz;
    }
    if (ntot > 2147483647LL || nztot > 2147483647LL) return -1;
  }
  auto h = std::make_unique<b200ldl_handle>();
  h->n = (int)ntot;
  h->nnz = (int)nztot;
  h->solver_type = solver_type;
  h->ustab = ustab;
  h->pivot_tol = pivot_tol;
  h->delay_growth = delay_growth;
  h->order = order;
  h->nsys = nsys;
  int st = guarded(h.get(), [&]() {
    std::vector<Symbolic> parts(nsys);
    std::vector<int> rowp_all(ntot + 1, 0), cols_all(nztot);
    long long ro = 0, co = 0, voff = 0;
    for (int si = 0; si < nsys; si++) {
      const int n = sys_n[si], nnz = sys_nnz[si];
      const int* rowp = rowp_cat + ro;
      const int* cols = cols_cat + co;
      parts[si] = analyze(static_cast<Ordering>(order), n, rowp, cols);
      for (int i = 0; i < n; i++) rowp_all[voff + i + 1] = (int)(co + rowp[i + 1]);
      for (int e = 0; e < nnz; e++) cols_all[co + e] = (int)(voff + cols[e]);
      ro += n + 1;
      co += nnz;
      voff += n;
    }
    h->sym = merge_symbolic(parts, h->node_sys);
    build_plan(h.get(), rowp_all.data(), cols_all.data());
    h->h_rowp = std::move(rowp_all);
    h->h_cols = std::move(cols_all);
    return 0;
  });
  if (st != 0) {
    std::fprintf(stderr, "b200ldl_create_batch: %s\n", h->last_error.c_str());
    return st;
  }
  *out = h.release();
  return 0;
}

int b200ldl_num_systems(b200ldl_t h) { return h ? h->nsys : -1; }

int b200ldl_value_gradient(b200ldl_t h, int nrhs, const double* lam, int ldl, const double* x,
                           int ldx, double* gvals, double* gdiag) {
  return guarded(h, [&]() {
    if (nrhs < 0 || nrhs > refine_max_rhs() || ldl < h->n || ldx < h->n ||
        (nrhs > 0 && (!lam || !x || (h->nnz > 0 && !gvals))))
      return fail(h, -1, "bad gradient arguments");
    if (h->n == 0) return 0;
    upload_plan(h);
    launch_value_gradient(h->n, h->d_rowp.ptr, h->d_cols.ptr, lam, ldl, x, ldx, nrhs, gvals,
                          gdiag, h->stream);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return 0;
  });
}

int b200ldl_system_inertia(b200ldl_t h, int* npos, int* nneg) {
  if (!h || !npos || !nneg) return -1;
  if (!h->factored) return fail(h, -5, "inertia requested before a successful factor");
  if (h->nsys == 1) {
    npos[0] = h->inertia[0];
    nneg[0] = h->inertia[1];
    return 0;
  }
  for (int si = 0; si < h->nsys; si++) {
    const bool have = h->sys_inertia.size() == (size_t)2 * h->nsys;
    npos[si] = have ? h->sys_inertia[2 * si] : 0;
    nneg[si] = have ? h->sys_inertia[2 * si + 1] : 0;
  }
  return 0;
}

void b200ldl_destroy(b200ldl_t h) { delete h; }

int b200ldl_set_stream(b200ldl_t h, void* stream) {
  if (!h) return -1;
  h->stream = static_cast<cudaStream_t>(stream);
  return 0;
}

int b200ldl_factor(b200ldl_t h, const double* vals, const double* diag) {
  return guarded(h, [&]() {
    if (h->nnz > 0 && !vals) return fail(h, -1, "vals is null");
    h->factored = false;
    h->fmax = 0;
    run_factor(h, vals, diag);
    return 0;
  });
}

int b200ldl_factor_elements(b200ldl_t h, b200ldl_assembly_t a, const double* blocks,
                            const double* diag) {
  return guarded(h, [&]() {
    int an = 0, annz = 0;
    const long long *aptr = nullptr, *asrc = nullptr;
    if (!a || assembly_device_plan(a, &an, &annz, &aptr, &asrc) != 0)
      return fail(h, -1, "no assembly plan");
    if (an != h->n || annz != h->nnz)
      return fail(h, -1,
                  "the assembly plan is for another pattern (n %d nnz %d, handle n %d nnz %d)",
                  an, annz, h->n, h->nnz);
    if (h->nnz > 0 && !blocks) return fail(h, -1, "blocks is null");
    if (h->precision != B200LDL_FP64)
      return fail(h, -1,
                  "element-block factorization needs the FP64 mode (the mixed mode refines "
                  "against CSR values)");
    // the source holds for this factorization only, whatever happens in it
    struct Source {
      b200ldl_t h;
      ~Source() {
        h->asm_ptr = h->asm_src = nullptr;
        h->asm_blocks = nullptr;
        h->st.asm_ptr = h->st.asm_src = nullptr;
        h->st.asm_blocks = nullptr;
      }
    } source{h};
    h->asm_ptr = h->st.asm_ptr = aptr;
    h->asm_src = h->st.asm_src = asrc;
    h->asm_blocks = h->st.asm_blocks = blocks;
    h->factored = false;
    h->fmax = 0;
    run_factor(h, nullptr, diag);
    return 0;
  });
}

int b200ldl_factor_host(b200ldl_t h, const double* vals, const double* diag) {
  return guarded(h, [&]() {
    if (h->nnz > 0 && !vals) return fail(h, -1, "vals is null");
    if (h->d_vals.count < (size_t)std::max(1, h->nnz)) CK(h->d_vals.alloc(h->nnz));
    CK(cudaMemcpyAsync(h->d_vals.ptr, vals, sizeof(double) * h->nnz, cudaMemcpyHostToDevice,
                       h->stream));
    const double* dd = nullptr;
    if (diag) {
      if (h->d_diag.count < (size_t)std::max(1, h->n)) CK(h->d_diag.alloc(h->n));
      CK(cudaMemcpyAsync(h->d_diag.ptr, diag, sizeof(double) * h->n, cudaMemcpyHostToDevice,
                         h->stream));
      dd = h->d_diag.ptr;
    }
    h->factored = false;
    h->fmax = 0;
    run_factor(h, h->d_vals.ptr, dd);
    return 0;
  });
}

int b200ldl_set_perturbation_rows(b200ldl_t h, int nprimal, const int* primal, int ndual,
                                  const int* dual) {
  return guarded(h, [&]() {
    if (nprimal < 0 || ndual < 0 || (nprimal > 0 && !primal) || (ndual > 0 && !dual))
      return fail(h, -1, "bad perturbation row lists");
    std::vector<unsigned char> cls(std::max(1, h->n), 0);
    for (int t = 0; t < nprimal; t++) {
      const int i = primal[t];
      if (i < 0 || i >= h->n) return fail(h, -1, "primal row index out of range");
      if (cls[i] & 1) return fail(h, -1, "primal row listed twice");
      cls[i] |= 1;
    }
    for (int t = 0; t < ndual; t++) {
      const int i = dual[t];
      if (i < 0 || i >= h->n) return fail(h, -1, "constraint row index out of range");
      if (cls[i] & 2) return fail(h, -1, "constraint row listed twice");
      cls[i] |= 2;
    }
    if (h->d_pclass.count < cls.size()) CK(h->d_pclass.alloc(cls.size()));
    if (h->d_pdiag.count < cls.size()) CK(h->d_pdiag.alloc(cls.size()));
    CK(cudaMemcpyAsync(h->d_pclass.ptr, cls.data(), cls.size(), cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->have_pclass = true;
    return 0;
  });
}

int b200ldl_factor_perturbed(b200ldl_t h, const double* vals, const double* diag,
                             double delta_x, double delta_c, int* npos, int* nneg) {
  return guarded(h, [&]() {
    if (h->nnz > 0 && !vals) return fail(h, -1, "vals is null");
    if (!h->have_pclass) return fail(h, -1, "perturbation rows not set");
    if (!(delta_x >= 0.0) || !(delta_c >= 0.0) || std::isinf(delta_x) || std::isinf(delta_c))
      return fail(h, -1, "perturbations must be finite and non-negative");
    h->factored = false;
    h->fmax = 0;
    if (h->n > 0)
      launch_perturb_diag(h->n, diag, h->d_pclass.ptr, delta_x, delta_c, h->d_pdiag.ptr,
                          h->stream);
    run_factor(h, vals, h->d_pdiag.ptr);
    if (npos) *npos = h->inertia[0];
    if (nneg) *nneg = h->inertia[1];
    return 0;
  });
}

int b200ldl_copy_perturbed_diagonal(b200ldl_t h, double* out) {
  return guarded(h, [&]() {
    if (!out) return fail(h, -1, "out is null");
    if (!h->have_pclass) return fail(h, -1, "perturbation rows not set");
    if (h->n > 0)
      CK(cudaMemcpyAsync(out, h->d_pdiag.ptr, sizeof(double) * h->n, cudaMemcpyDeviceToDevice,
                         h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return 0;
  });
}

// In place x <- K^-1 x for device x. After a mixed-precision factorization
// the solution is refined in FP64 against the matrix that was factored.
static void solve_inplace(b200ldl_t h, int nrhs, double* x, int ldx) {
  if (h->factored_mixed && h->nnz > 0 && h->last_vals) {
    const size_t cnt = (size_t)h->n * nrhs;
    if (h->d_rhs_tmp.count < cnt) CK(h->d_rhs_tmp.alloc(cnt));
    launch_copy_cols(h->n, nrhs, x, ldx, h->d_rhs_tmp.ptr, h->n, h->stream);
    refine_impl(h, h->last_vals, h->last_diag, nrhs, h->d_rhs_tmp.ptr, h->n, x, ldx,
                h->refine_max, h->refine_tol, nullptr, nullptr);
    if (h->last_berr <= h->refine_tol) return;
    // refinement stalled on the mixed factor: factor in FP64 and solve again
    h->mixed_fallbacks++;
    run_factor_once(h, h->last_vals, h->last_diag, false);
    h->fmax = 0;
    launch_copy_cols(h->n, nrhs, h->d_rhs_tmp.ptr, h->n, x, ldx, h->stream);
  }
  run_solve(h, nrhs, x, ldx);
  CK(cudaStreamSynchronize(h->stream));
  h->prof.collect();
}

int b200ldl_solve(b200ldl_t h, int nrhs, double* x, int ldx) {
  return guarded(h, [&]() {
    if (!h->factored) return fail(h, -5, "solve called before a successful factor");
    if (nrhs < 0 || ldx < h->n || (nrhs > 0 && !x)) return fail(h, -1, "bad solve arguments");
    if (nrhs == 0 || h->n == 0) return 0;
    solve_inplace(h, nrhs, x, ldx);
    return 0;
  });
}

int b200ldl_set_precision(b200ldl_t h, int mode) {
  if (!h) return -1;
  if (mode != B200LDL_FP64 && mode != B200LDL_MIXED) return fail(h, -1, "unknown precision mode");
  h->precision = mode;
  return 0;
}

int b200ldl_set_refinement(b200ldl_t h, int max_iter, double tol) {
  if (!h) return -1;
  if (max_iter < 0 || !(tol >= 0.0)) return fail(h, -1, "bad refinement settings");
  h->refine_max = max_iter;
  h->refine_tol = tol;
  return 0;
}

int b200ldl_last_refinement(b200ldl_t h, int* iters, double* berr, int* mixed,
                            int* fallbacks) {
  if (!h) return -1;
  if (iters) *iters = h->last_iters;
  if (berr) *berr = h->last_berr;
  if (mixed) *mixed = h->factored_mixed ? 1 : 0;
  if (fallbacks) *fallbacks = h->mixed_fallbacks;
  return 0;
}

int b200ldl_solve_host(b200ldl_t h, int nrhs, double* x, int ldx) {
  return guarded(h, [&]() {
    if (!h->factored) return fail(h, -5, "solve called before a successful factor");
    if (nrhs < 0 || ldx < h->n || (nrhs > 0 && !x)) return fail(h, -1, "bad solve arguments");
    if (nrhs == 0 || h->n == 0) return 0;
    const size_t cnt = (size_t)ldx * nrhs;
    if (h->d_x.count < cnt) CK(h->d_x.alloc(cnt));
    CK(cudaMemcpyAsync(h->d_x.ptr, x, cnt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    solve_inplace(h, nrhs, h->d_x.ptr, ldx);
    CK(cudaMemcpyAsync(x, h->d_x.ptr, cnt * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->prof.collect();
    return 0;
  });
}

int b200ldl_get_inertia(b200ldl_t h, int* npos, int* nneg) {
  if (!h || !npos || !nneg) return -1;
  if (!h->factored) return fail(h, -5, "inertia requested before a successful factor");
  *npos = h->inertia[0];
  *nneg = h->inertia[1];
  return 0;
}

const char* b200ldl_last_error(b200ldl_t h) { return h ? h->last_error.c_str() : "null handle"; }

int b200ldl_symbolic_sizes(b200ldl_t h, int* num_nodes, int* num_contrib) {
  if (!h) return -1;
  if (num_nodes) *num_nodes = h->sym.num_nodes;
  if (num_contrib) *num_contrib = (int)h->sym.contrib_rows.size();
  return 0;
}

int b200ldl_get_symbolic(b200ldl_t h, int* invperm, int* node_ptr, int* node_to_var,
                         int* children_ptr, int* children, int* contrib_ptr,
                         int* contrib_rows) {
  if (!h) return -1;
  const Symbolic& s = h->sym;
  auto cp = [](const std::vector<int>& v, int* dst) {
    if (dst) std::copy(v.begin(), v.end(), dst);
  };
  if (invperm) {
    for (int i = 0; i < s.n; i++) invperm[i] = s.permuted ? s.iperm[i] : i;
  }
  cp(s.node_ptr, node_ptr);
  cp(s.node_to_var, node_to_var);
  cp(s.children_ptr, children_ptr);
  if (children) std::copy(s.children.begin(), s.children.begin() + s.num_nodes, children);
  cp(s.contrib_ptr, contrib_ptr);
  cp(s.contrib_rows, contrib_rows);
  return 0;
}

int b200ldl_node_pivots(b200ldl_t h, int* num_pivots, int* num_delayed) {
  return guarded(h, [&]() {
    if (!h->factored) return fail(h, -5, "no factorization");
    const int nn = h->sym.num_nodes;
    if (num_pivots) CK(cudaMemcpy(num_pivots, h->d_npiv.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
    if (num_delayed) CK(cudaMemcpy(num_delayed, h->d_ndel.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
    return 0;
  });
}

int b200ldl_get_pivot_record(b200ldl_t h, int* f, int* npiv, int* ndel, int* fv,
                             long long* fv_len) {
  return guarded(h, [&]() {
    if (!h->factored) return fail(h, -5, "no factorization");
    const int nn = h->sym.num_nodes;
    std::vector<int> hf(nn), hp(nn), hd(nn);
    std::vector<int64_t> ho(nn);
    if (nn > 0) {
      CK(cudaMemcpy(hf.data(), h->d_f.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(hp.data(), h->d_npiv.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(hd.data(), h->d_ndel.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
      CK(cudaMemcpy(ho.data(), h->d_fv_off.ptr, nn * sizeof(int64_t), cudaMemcpyDeviceToHost));
    }
    long long total = 0;
    for (int k = 0; k < nn; k++) total += hf[k];
    if (fv_len) *fv_len = total;
    if (f) std::copy(hf.begin(), hf.end(), f);
    if (npiv) std::copy(hp.begin(), hp.end(), npiv);
    if (ndel) std::copy(hd.begin(), hd.end(), ndel);
    if (fv && total > 0) {
      std::vector<int> pool(h->used[0]);
      CK(cudaMemcpy(pool.data(), h->d_ivars.ptr, pool.size() * sizeof(int),
                    cudaMemcpyDeviceToHost));
      long long o = 0;
      for (int k = 0; k < nn; k++) {
        if (ho[k] < 0 || (unsigned long long)(ho[k] + hf[k]) > h->used[0])
          return fail(h, -4, "front variables of supernode %d outside the used pool", k);
        std::copy(pool.begin() + ho[k], pool.begin() + ho[k] + hf[k], fv + o);
        o += hf[k];
      }
    }
    return 0;
  });
}

int b200ldl_set_pivot_record(b200ldl_t h, const int* f, const int* npiv, const int* ndel,
                             const int* fv) {
  return guarded(h, [&]() {
    if (h->solver_type == B200LDL_CHOLESKY) return fail(h, -1, "Cholesky mode has no pivot order");
    if (!f && !npiv && !ndel && !fv) {
      if (h->replanned) {
        h->replanned = false;
        try {
          use_structure(h, Symbolic(h->sym_ref));
        } catch (...) {
          h->replanned = true;
          throw;
        }
      }
      return 0;
    }
    if (!f || !npiv || !ndel || !fv) return fail(h, -1, "incomplete pivot record");
    if (!h->replanned) h->sym_ref = h->sym;
    std::vector<int> partner(std::max(1, h->n), -1);
    Symbolic s = replan_from_record(h->sym_ref, f, npiv, ndel, fv, partner);
    const bool was = h->replanned;
    h->replanned = true;
    try {
      use_structure(h, std::move(s));
    } catch (...) {
      h->replanned = was;
      throw;
    }
    h->partner = std::move(partner);
    return 0;
  });
}

int b200ldl_reuse_pivot_order(b200ldl_t h) {
  if (!h) return -1;
  const int nn = h->sym.num_nodes;
  long long total = 0;
  int st = b200ldl_get_pivot_record(h, nullptr, nullptr, nullptr, nullptr, &total);
  if (st != 0) return st;
  std::vector<int> f(std::max(1, nn)), np(std::max(1, nn)), nd(std::max(1, nn));
  std::vector<int> fv(std::max<long long>(1, total));
  st = b200ldl_get_pivot_record(h, f.data(), np.data(), nd.data(), fv.data(), &total);
  if (st != 0) return st;
  return b200ldl_set_pivot_record(h, f.data(), np.data(), nd.data(), fv.data());
}

int b200ldl_stats(b200ldl_t h, double* stats, int nstats) {
  return guarded(h, [&]() {
    if (!h->factored) return fail(h, -5, "no factorization");
    const int nn = h->sym.num_nodes;
    std::vector<int> f(nn), np(nn), nd(nn);
    CK(cudaMemcpy(f.data(), h->d_f.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(np.data(), h->d_npiv.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(nd.data(), h->d_ndel.ptr, nn * sizeof(int), cudaMemcpyDeviceToHost));
    double lbytes = 0, cbytes = 0, sdel = 0;
    int fm = 0;
    for (int k = 0; k < nn; k++) {
      lbytes += 8.0 * f[k] * np[k];
      cbytes += 8.0 * (double)(f[k] - np[k]) * (f[k] - np[k]);
      sdel += nd[k];
      fm = std::max(fm, f[k]);
    }
    const double v[6] = {h->exec_flops, lbytes, cbytes, (double)fm, sdel, (double)h->num_levels};
    for (int i = 0; i < nstats && i < 6; i++) stats[i] = v[i];
    return 0;
  });
}

int b200ldl_solve_refine(b200ldl_t h, const double* vals, const double* diag, int nrhs,
                         const double* b, int ldb, double* x, int ldx, int max_iter, double tol,
                         double* berr_out, int* iters_out) {
  return guarded(h, [&]() {
    if (!h->factored) return fail(h, -5, "solve called before a successful factor");
    if (nrhs < 0 || ldb < h->n || ldx < h->n || max_iter < 0 || (nrhs > 0 && (!b || !x)) ||
        (h->nnz > 0 && !vals))
      return fail(h, -1, "bad refine arguments");
    refine_impl(h, vals, diag, nrhs, b, ldb, x, ldx, max_iter, tol, berr_out, iters_out);
    return 0;
  });
}

int b200ldl_set_profiling(b200ldl_t h, int enable) {
  if (!h) return -1;
  h->prof.on = enable != 0;
  return 0;
}

int b200ldl_reset_profile(b200ldl_t h) {
  if (!h) return -1;
  h->prof.reset();
  return 0;
}

int b200ldl_profile(b200ldl_t h, double* out, int n) {
  if (!h || !out) return -1;
  for (int p = 0; p < kPhN && 2 * p + 1 < n; p++) {
    out[2 * p] = h->prof.ms[p];
    out[2 * p + 1] = (double)h->prof.launches[p];
  }
  return 0;
}

long long b200ldl_launch_count(b200ldl_t h) { return h ? h->prof.total_launches : -1; }

int b200ldl_work(b200ldl_t h, double* out, int n) {
  if (!h || !out) return -1;
  for (int i = 0; i < kWork && i < n; i++) out[i] = h->flops4[i];
  return 0;
}

}  // extern "C"
