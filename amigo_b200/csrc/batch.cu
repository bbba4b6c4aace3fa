// Many independent KKT systems factored and solved as one forest.
//
// Each system keeps its own symbolic phase (the reference's ordering,
// elimination tree and supernodes, bit for bit, as if it were factored
// alone); the plans are concatenated into one forest, so every level of the
// numeric factorization and of the solve runs the fronts of all systems in
// the same launches. The inertia of each system is read back from the
// stored D blocks, with the reference's rule (SparseLDL::add_pivot_inertia,
// include/sparse_ldl.h:1935-1987): a 1x1 pivot counts by its sign (zero as
// positive), a 2x2 block with det >= 0 twice by the sign of d11, a 2x2 block
// with det < 0 once each way.
#include <stdexcept>

#include "ldl_internal.h"
#include "symbolic.h"

namespace b200ldl {

namespace {

// one warp per supernode; 2x2 pairs are consecutive 2x2-marked positions
// starting at a run's first position
__global__ void system_inertia_kernel(DevState s, const int* __restrict__ node_sys, int nn,
                                      int* __restrict__ sys_inertia) {
  const int lane = threadIdx.x & 31;
  const int node = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (node >= nn) return;
  const int npiv = s.npiv[node];
  const int* fv = s.ivars + s.fv_off[node];
  const double* L = s.dpool + s.L_off[node];
  const int ldl = s.L_ld[node];
  int pos = 0, neg = 0;
  int carry = 0;  // parity of the 2x2 run length entering the chunk
  for (int w = 0; w * 32 < npiv; w++) {
    const int p = 32 * w + lane;
    const bool mark = p < npiv && fv[p] < 0;
    const unsigned mm = __ballot_sync(0xffffffffu, mark);
    const unsigned below = (~mm) & ((1u << lane) - 1u);
    const int ridx = below ? lane - 32 + __clz(below) : lane + carry;
    if (p < npiv) {
      if (!mark) {
        if (L[p + (size_t)ldl * p] >= 0.0)
          pos++;
        else
          neg++;
      } else if ((ridx & 1) == 0) {  // first row of a 2x2 block
        const double d11 = L[p + (size_t)ldl * p];
        const double d21 = L[(p + 1) + (size_t)ldl * p];
        const double d22 = L[(p + 1) + (size_t)ldl * (p + 1)];
        const double det = d11 * d22 - d21 * d21;
        if (det >= 0.0) {
          if (d11 >= 0.0)
            pos += 2;
          else
            neg += 2;
        } else {
          pos++;
          neg++;
        }
      }
    }
    const int r31 = __shfl_sync(0xffffffffu, ridx, 31);
    carry = ((mm >> 31) & 1u) ? ((r31 + 1) & 1) : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    pos += __shfl_xor_sync(0xffffffffu, pos, o);
    neg += __shfl_xor_sync(0xffffffffu, neg, o);
  }
  if (lane == 0 && (pos | neg)) {
    const int sy = node_sys[node];
    atomicAdd(sys_inertia + 2 * sy, pos);
    atomicAdd(sys_inertia + 2 * sy + 1, neg);
  }
}

}  // namespace

void launch_system_inertia(const DevState& s, const int* node_sys, int nn, int* sys_inertia,
                           cudaStream_t st) {
  if (nn <= 0) return;
  const int threads = 256;
  const int blocks = (int)(((long long)nn * 32 + threads - 1) / threads);
  system_inertia_kernel<<<blocks, threads, 0, st>>>(s, node_sys, nn, sys_inertia);
}

// Concatenate per-system symbolic results: variables, nodes and contribution
// rows shifted by the systems before; roots of every system at the end.
Symbolic merge_symbolic(const std::vector<Symbolic>& parts, std::vector<int>& node_sys) {
  Symbolic m;
  int n = 0, nn = 0;
  size_t ncontrib = 0;
  for (const Symbolic& p : parts) {
    n += p.n;
    nn += p.num_nodes;
    ncontrib += p.contrib_rows.size();
    m.permuted = m.permuted || p.permuted;
  }
  m.n = n;
  m.num_nodes = nn;
  m.perm.resize(n);
  m.iperm.resize(n);
  m.node_ptr.assign(nn + 1, 0);
  m.node_to_var.resize(n);
  m.children_ptr.assign(nn + 2, 0);
  m.children.reserve(nn);
  m.contrib_ptr.assign(nn + 1, 0);
  m.contrib_rows.reserve(ncontrib);
  m.parent.resize(nn);
  node_sys.resize(nn);
  int voff = 0, noff = 0;
  for (size_t si = 0; si < parts.size(); si++) {
    const Symbolic& p = parts[si];
    for (int k = 0; k < p.n; k++) {
      m.perm[voff + k] = voff + p.perm[k];
      m.iperm[voff + k] = voff + p.iperm[k];
      m.node_to_var[voff + k] = voff + p.node_to_var[k];
    }
    for (int k = 0; k < p.num_nodes; k++) {
      m.node_ptr[noff + k + 1] = voff + p.node_ptr[k + 1];
      m.children_ptr[noff + k] = (int)m.children.size();
      for (int c = p.children_ptr[k]; c < p.children_ptr[k + 1]; c++)
        m.children.push_back(noff + p.children[c]);
      m.contrib_ptr[noff + k] = (int)m.contrib_rows.size();
      for (int t = p.contrib_ptr[k]; t < p.contrib_ptr[k + 1]; t++)
        m.contrib_rows.push_back(voff + p.contrib_rows[t]);
      m.parent[noff + k] = p.parent[k] < 0 ? -1 : noff + p.parent[k];
      node_sys[noff + k] = (int)si;
    }
    voff += p.n;
    noff += p.num_nodes;
  }
  m.contrib_ptr[nn] = (int)m.contrib_rows.size();
  m.children_ptr[nn] = (int)m.children.size();
  noff = 0;
  for (const Symbolic& p : parts) {
    for (int c = p.children_ptr[p.num_nodes]; c < p.children_ptr[p.num_nodes + 1]; c++)
      m.children.push_back(noff + p.children[c]);
    noff += p.num_nodes;
  }
  m.children_ptr[nn + 1] = (int)m.children.size();
  if ((int)m.children.size() != nn) throw std::runtime_error("merged forest is inconsistent");
  return m;
}

}  // namespace b200ldl
