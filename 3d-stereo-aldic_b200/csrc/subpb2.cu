// ALDIC's global step, Subpb2Quadtree (func_quadtree/Subpb2Quadtree.m), on the device.
//
// On a quadtree mesh of 8-node elements (corners 1-4; mid-side "hanging" nodes 5-8 where a
// neighbour is refined, 0 where absent) the step minimises, in the finite-element space,
//   sum over elements and Gauss points of |J| w ((beta + alpha) |grad Uhat|^2
//       - 2 beta grad(N_a) . F_a Uhat_a + mu |Uhat - U|^2 + alpha grad(N) U terms)
// i.e. it solves A Uhat = b with (:149-204)
//   A_e = sum_g |J| w ((beta + alpha) DN' DN + mu N' N),
//   b_e = sum_g |J| w (beta diag(DN' F_rows') + mu N' N U_e + alpha DN' DN U_e),
// where the F rows of an x dof of node a are (F11_a, F12_a) and of a y dof (F21_a, F22_a), and
// v, W are 0 (:40-41: 0 * vdual, 0 * udual).  Both DN' DN and N' N couple x dofs with x dofs
// and y with y by the same numbers, so A_e = K_e (x) I_2 with one 8 x 8 K_e per element, and
// the x and y systems share one matrix.
//
// Layout: K_e row-major per element (64 doubles), b_e per element as (x, y) per local node
// (16 doubles); node -> (element, slot) adjacency lists built on the host, so every product
// and right-hand side is a gather in a fixed order (deterministic, no atomics).  The free
// nodes (all nodes of the elements but the first of unique(elementsFEM), :234-238, less
// the dirichlet nodes) are solved by Jacobi-preconditioned conjugate gradients on the
// interleaved 2 n vector; the dirichlet nodes hold U (:271-273) and enter the right-hand
// side through the same gather.  The reference solves the free block directly (:276).
#include <algorithm>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "kernels.h"

namespace aldic {

// Gauss points and weights of :60-77 (orders 4 and 5 with the file's rounded constants).
struct GaussRule {
  int np;
  double pt[5];
  double wt[5];
};

__host__ __device__ inline GaussRule gauss_rule(int order) {
  GaussRule g{};
  if (order == 2) {
    g.np = 2;
    g.pt[0] = -1.0 / sqrt(3.0);
    g.pt[1] = 1.0 / sqrt(3.0);
    g.wt[0] = g.wt[1] = 1.0;
  } else if (order == 3) {
    g.np = 3;
    g.pt[0] = 0.0;
    g.pt[1] = sqrt(3.0 / 5.0);
    g.pt[2] = -sqrt(3.0 / 5.0);
    g.wt[0] = 8.0 / 9.0;
    g.wt[1] = g.wt[2] = 5.0 / 9.0;
  } else if (order == 4) {
    g.np = 4;
    g.pt[0] = 0.339981;
    g.pt[1] = -0.339981;
    g.pt[2] = 0.861136;
    g.pt[3] = -0.861136;
    g.wt[0] = g.wt[1] = 0.652145;
    g.wt[2] = g.wt[3] = 0.347855;
  } else {
    g.np = 5;
    g.pt[0] = 0.0;
    g.pt[1] = 0.538469;
    g.pt[2] = -0.538469;
    g.pt[3] = 0.90618;
    g.pt[4] = -0.90618;
    g.wt[0] = 0.568889;
    g.wt[1] = g.wt[2] = 0.478629;
    g.wt[3] = g.wt[4] = 0.236927;
  }
  return g;
}

__host__ __device__ inline double sgn(double x) { return (double)((x > 0.0) - (x < 0.0)); }

// Shape functions and their (ksi, eta) derivatives (:138-148 and funDN*, :343-396): the
// corner functions less half of the two adjacent mid-side ones; d5..d8 switch the mid-side
// nodes (right, top, left, bottom edge) on; sign(0) = 0 as MATLAB's.
__host__ __device__ inline void quadtree_shape(double ksi, double eta, const double d[4], double N[8],
                                               double dk[8], double de[8]) {
  const double aks = fabs(ksi), aet = fabs(eta);
  N[4] = d[0] * 0.5 * (1.0 + ksi) * (1.0 - aet);
  N[5] = d[1] * 0.5 * (1.0 + eta) * (1.0 - aks);
  N[6] = d[2] * 0.5 * (1.0 - ksi) * (1.0 - aet);
  N[7] = d[3] * 0.5 * (1.0 - eta) * (1.0 - aks);
  N[0] = (1.0 - ksi) * (1.0 - eta) * 0.25 - 0.5 * (N[6] + N[7]);
  N[1] = (1.0 + ksi) * (1.0 - eta) * 0.25 - 0.5 * (N[7] + N[4]);
  N[2] = (1.0 + ksi) * (1.0 + eta) * 0.25 - 0.5 * (N[4] + N[5]);
  N[3] = (1.0 - ksi) * (1.0 + eta) * 0.25 - 0.5 * (N[5] + N[6]);
  dk[4] = d[0] * 0.5 * (1.0 - aet);
  de[4] = d[0] * 0.5 * (1.0 + ksi) * sgn(-eta);
  dk[5] = d[1] * 0.5 * (1.0 + eta) * sgn(-ksi);
  de[5] = d[1] * 0.5 * (1.0 - aks);
  dk[6] = d[2] * 0.5 * (-1.0) * (1.0 - aet);
  de[6] = d[2] * 0.5 * (1.0 - ksi) * sgn(-eta);
  dk[7] = d[3] * 0.5 * (1.0 - eta) * sgn(-ksi);
  de[7] = d[3] * 0.5 * (-1.0) * (1.0 - aks);
  dk[0] = -0.25 * (1.0 - eta) - 0.5 * (dk[6] + dk[7]);
  de[0] = -0.25 * (1.0 - ksi) - 0.5 * (de[6] + de[7]);
  dk[1] = 0.25 * (1.0 - eta) - 0.5 * (dk[7] + dk[4]);
  de[1] = -0.25 * (1.0 + ksi) - 0.5 * (de[7] + de[4]);
  dk[2] = 0.25 * (1.0 + eta) - 0.5 * (dk[4] + dk[5]);
  de[2] = 0.25 * (1.0 + ksi) - 0.5 * (de[4] + de[5]);
  dk[3] = -0.25 * (1.0 + eta) - 0.5 * (dk[5] + dk[6]);
  de[3] = 0.25 * (1.0 - ksi) - 0.5 * (de[5] + de[6]);
}

// Row a of K_e and the (x, y) right-hand side of local node a of one element.  xy: the 8
// nodes' coordinates (0 at absent mid-side nodes, as the reference), ue: their (x, y)
// displacements U (0 when absent), fa: node a's (F11, F21, F12, F22).
__host__ __device__ inline void subpb2_element_row(int a, const double xy[16], const double d[4], const double ue[16],
                                                   const double fa[4], int order, double beta, double mu,
                                                   double alpha, double krow[8], double brow[2]) {
  const GaussRule g = gauss_rule(order);
  for (int b = 0; b < 8; ++b) krow[b] = 0.0;
  brow[0] = brow[1] = 0.0;
  for (int je = 0; je < g.np; ++je)    // ndgrid order: ksi runs fastest
    for (int ik = 0; ik < g.np; ++ik) {
      const double ksi = g.pt[ik], eta = g.pt[je], w = g.wt[ik] * g.wt[je];
      double N[8], dk[8], de[8];
      quadtree_shape(ksi, eta, d, N, dk, de);
      double j11 = 0.0, j12 = 0.0, j21 = 0.0, j22 = 0.0;
      for (int k = 0; k < 8; ++k) {
        j11 += dk[k] * xy[2 * k];
        j12 += dk[k] * xy[2 * k + 1];
        j21 += de[k] * xy[2 * k];
        j22 += de[k] * xy[2 * k + 1];
      }
      const double jac = j11 * j22 - j12 * j21;
      const double i11 = j22 / jac, i12 = -j12 / jac, i21 = -j21 / jac, i22 = j11 / jac;
      const double jw = jac * w;
      const double dxa = i11 * dk[a] + i12 * de[a], dya = i21 * dk[a] + i22 * de[a];
      double mux = 0.0, muy = 0.0, alx = 0.0, aly = 0.0;
      for (int b = 0; b < 8; ++b) {
        const double dxb = i11 * dk[b] + i12 * de[b], dyb = i21 * dk[b] + i22 * de[b];
        const double gg = dxa * dxb + dya * dyb, nn = N[a] * N[b];
        krow[b] += jw * ((beta + alpha) * gg + mu * nn);
        mux += nn * ue[2 * b];
        muy += nn * ue[2 * b + 1];
        alx += gg * ue[2 * b];
        aly += gg * ue[2 * b + 1];
      }
      brow[0] += jw * (beta * (dxa * fa[0] + dya * fa[2]) + mu * mux + alpha * alx);
      brow[1] += jw * (beta * (dxa * fa[1] + dya * fa[3]) + mu * muy + alpha * aly);
    }
}

// One thread per (element, local node): K_e row and b_e entries; rows of absent nodes are 0.
// elem: n_el x 8 column-major, 1-based node numbers (0 = no mid-side node); coords n x 2
// column-major; U 2n interleaved; F 4n (F11 F21 F12 F22 per node).
__global__ void subpb2_element_kernel(int n_el, const int* __restrict__ elem, const double* __restrict__ coords,
                                      long long n, const double* __restrict__ U, const double* __restrict__ F,
                                      int order, double beta, double mu, double alpha, double* __restrict__ Ke,
                                      double* __restrict__ be) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= 8LL * n_el) return;
  const int e = (int)(t >> 3), a = (int)(t & 7);
  double* kr = Ke + (long long)e * 64 + a * 8;
  double* br = be + (long long)e * 16 + a * 2;
  int id[8];
  for (int k = 0; k < 8; ++k) id[k] = elem[e + (long long)k * n_el];
  if (id[a] == 0) {
    for (int b = 0; b < 8; ++b) kr[b] = 0.0;
    br[0] = br[1] = 0.0;
    return;
  }
  double xy[16], ue[16], d[4], fa[4];
  for (int k = 0; k < 8; ++k) {
    const long long g = id[k] - 1;
    const bool on = id[k] != 0;
    xy[2 * k] = on ? coords[g] : 0.0;
    xy[2 * k + 1] = on ? coords[g + n] : 0.0;
    ue[2 * k] = on ? U[2 * g] : 0.0;
    ue[2 * k + 1] = on ? U[2 * g + 1] : 0.0;
  }
  for (int k = 0; k < 4; ++k) d[k] = id[4 + k] != 0 ? 1.0 : 0.0;
  const long long ga = id[a] - 1;
  for (int k = 0; k < 4; ++k) fa[k] = F[4 * ga + k];
  double krow[8], brow[2];
  subpb2_element_row(a, xy, d, ue, fa, order, beta, mu, alpha, krow, brow);
  for (int b = 0; b < 8; ++b) kr[b] = krow[b];
  br[0] = brow[0];
  br[1] = brow[1];
}

// (K x) at node i for both components: the node's (element, slot) entries, each a row of
// that element's K_e against the element's nodes.  x is 2n interleaved.
__host__ __device__ inline void subpb2_gather_row(long long i, const int* adj_ptr, const int* adj, const int* elem,
                                                  int n_el, const double* Ke, const double* x, double& yx,
                                                  double& yy) {
  yx = 0.0;
  yy = 0.0;
  for (int q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
    const int e = adj[q] >> 3, s = adj[q] & 7;
    const double* kr = Ke + (long long)e * 64 + s * 8;
    for (int b = 0; b < 8; ++b) {
      const int nb = elem[e + (long long)b * n_el];
      if (nb == 0) continue;
      yx += kr[b] * x[2 * (long long)(nb - 1)];
      yy += kr[b] * x[2 * (long long)(nb - 1) + 1];
    }
  }
}

// CG scalars, one set for the interleaved 2 n system.
struct Subpb2Scalars {
  double rz, alpha, beta, rr0, rr;
  int it, done, ok;
};

namespace {

constexpr int kSubpb2Threads = 256;

__device__ __forceinline__ void block_partial(double v0, double v1, double* part) {
  __shared__ double red[2][kSubpb2Threads / 32];
  v0 = warp_sum(v0);
  v1 = warp_sum(v1);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][wid] = v0;
    red[1][wid] = v1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0.0, s1 = 0.0;
    for (int k = 0; k < kSubpb2Threads / 32; ++k) {
      s0 += red[0][k];
      s1 += red[1][k];
    }
    part[2 * blockIdx.x] = s0;
    part[2 * blockIdx.x + 1] = s1;
  }
}

// Fixed-order sum of the per-block partials (one block).
__device__ __forceinline__ void sum_partials(const double* part, int nparts, double& s0, double& s1) {
  __shared__ double red[2][kSubpb2Threads];
  double a0 = 0.0, a1 = 0.0;
  for (int k = threadIdx.x; k < nparts; k += blockDim.x) {
    a0 += part[2 * k];
    a1 += part[2 * k + 1];
  }
  red[0][threadIdx.x] = a0;
  red[1][threadIdx.x] = a1;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0;
    for (int k = 0; k < (int)blockDim.x; ++k) {
      t0 += red[0][k];
      t1 += red[1][k];
    }
    s0 = t0;
    s1 = t1;
  }
}

}  // namespace

// b, the Jacobi diagonal and the start: x = U at dirichlet nodes (0 elsewhere), then (second
// kernel) r = b - K x, z = r / D, p = z on the free nodes.  free[i]: 1 free, 2 dirichlet, 0
// neither.
__global__ void subpb2_rhs_kernel(long long n, const int* __restrict__ adj_ptr, const int* __restrict__ adj,
                                  const double* __restrict__ Ke, const double* __restrict__ be,
                                  const unsigned char* __restrict__ free_, const double* __restrict__ U,
                                  double* __restrict__ b, double* __restrict__ D, double* __restrict__ x) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double bx = 0.0, by = 0.0, dg = 0.0;
  for (int q = adj_ptr[i]; q < adj_ptr[i + 1]; ++q) {
    const int e = adj[q] >> 3, s = adj[q] & 7;
    bx += be[(long long)e * 16 + 2 * s];
    by += be[(long long)e * 16 + 2 * s + 1];
    dg += Ke[(long long)e * 64 + s * 9];
  }
  b[2 * i] = bx;
  b[2 * i + 1] = by;
  D[i] = dg;
  const bool dir = free_[i] == 2;
  x[2 * i] = dir ? U[2 * i] : 0.0;
  x[2 * i + 1] = dir ? U[2 * i + 1] : 0.0;
}

__global__ void subpb2_start_kernel(long long n, const int* __restrict__ adj_ptr, const int* __restrict__ adj,
                                    const int* __restrict__ elem, int n_el, const double* __restrict__ Ke,
                                    const unsigned char* __restrict__ free_, const double* __restrict__ b,
                                    const double* __restrict__ D, const double* __restrict__ x,
                                    double* __restrict__ r, double* __restrict__ z, double* __restrict__ p,
                                    double* __restrict__ part) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double rz = 0.0, rr = 0.0;
  if (i < n) {
    double rx = 0.0, ry = 0.0, zx = 0.0, zy = 0.0;
    if (free_[i] == 1) {
      double kx, ky;
      subpb2_gather_row(i, adj_ptr, adj, elem, n_el, Ke, x, kx, ky);
      rx = b[2 * i] - kx;
      ry = b[2 * i + 1] - ky;
      zx = rx / D[i];
      zy = ry / D[i];
    }
    r[2 * i] = rx;
    r[2 * i + 1] = ry;
    z[2 * i] = zx;
    z[2 * i + 1] = zy;
    p[2 * i] = zx;
    p[2 * i + 1] = zy;
    rz = rx * zx + ry * zy;
    rr = rx * rx + ry * ry;
  }
  block_partial(rz, rr, part);
}

__global__ void subpb2_init_scalars_kernel(const double* __restrict__ part, int nparts, Subpb2Scalars* sc) {
  double rz, rr;
  sum_partials(part, nparts, rz, rr);
  if (threadIdx.x == 0) {
    sc->rz = rz;
    sc->rr0 = rr;
    sc->rr = rr;
    sc->it = 0;
    sc->ok = 1;
    sc->done = rr == 0.0 ? 1 : 0;
  }
}

// q = K p on the free nodes (0 elsewhere) and the partial p . q.
__global__ void subpb2_matvec_kernel(long long n, const int* __restrict__ adj_ptr, const int* __restrict__ adj,
                                     const int* __restrict__ elem, int n_el, const double* __restrict__ Ke,
                                     const unsigned char* __restrict__ free_, const double* __restrict__ p,
                                     double* __restrict__ q, double* __restrict__ part,
                                     const Subpb2Scalars* __restrict__ sc) {
  if (sc->done) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double pq = 0.0;
  if (i < n) {
    double qx = 0.0, qy = 0.0;
    if (free_[i] == 1) subpb2_gather_row(i, adj_ptr, adj, elem, n_el, Ke, p, qx, qy);
    q[2 * i] = qx;
    q[2 * i + 1] = qy;
    pq = p[2 * i] * qx + p[2 * i + 1] * qy;
  }
  block_partial(pq, 0.0, part);
}

__global__ void subpb2_alpha_kernel(const double* __restrict__ part, int nparts, Subpb2Scalars* sc) {
  if (sc->done) return;
  double pq, unused;
  sum_partials(part, nparts, pq, unused);
  if (threadIdx.x == 0) {
    if (!(pq > 0.0)) {  // no descent direction left: stop with what x holds
      sc->done = 1;
      sc->ok = 0;
    } else {
      sc->alpha = sc->rz / pq;
    }
  }
}

// x += alpha p, r -= alpha q, z = r / D on the free nodes; partials r . z and r . r.
__global__ void subpb2_update_kernel(long long n, const unsigned char* __restrict__ free_,
                                     const double* __restrict__ D, const double* __restrict__ p,
                                     const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r,
                                     double* __restrict__ z, double* __restrict__ part,
                                     const Subpb2Scalars* __restrict__ sc) {
  if (sc->done) return;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double rz = 0.0, rr = 0.0;
  if (i < n && free_[i] == 1) {
    const double al = sc->alpha;
    for (int c = 0; c < 2; ++c) {
      const long long k = 2 * i + c;
      x[k] += al * p[k];
      const double rn = r[k] - al * q[k];
      r[k] = rn;
      const double zn = rn / D[i];
      z[k] = zn;
      rz += rn * zn;
      rr += rn * rn;
    }
  }
  block_partial(rz, rr, part);
}

__global__ void subpb2_beta_kernel(const double* __restrict__ part, int nparts, double tol2, int maxit,
                                   Subpb2Scalars* sc) {
  if (sc->done) return;
  double rz, rr;
  sum_partials(part, nparts, rz, rr);
  if (threadIdx.x == 0) {
    sc->beta = rz / sc->rz;
    sc->rz = rz;
    sc->rr = rr;
    sc->it += 1;
    if (rr <= tol2 * sc->rr0 || sc->it >= maxit) sc->done = 1;
    if (sc->it >= maxit && rr > tol2 * sc->rr0) sc->ok = 0;
  }
}

// p = z + beta p (free nodes; p stays 0 elsewhere).  Runs after a converged step too: the
// extra update leaves x untouched.
__global__ void subpb2_direction_kernel(long long n, const unsigned char* __restrict__ free_,
                                        const double* __restrict__ z, double* __restrict__ p,
                                        const Subpb2Scalars* __restrict__ sc) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || free_[i] != 1) return;
  const double be = sc->beta;
  p[2 * i] = z[2 * i] + be * p[2 * i];
  p[2 * i + 1] = z[2 * i + 1] + be * p[2 * i + 1];
}

int subpb2_blocks(long long n) { return (int)((n + kSubpb2Threads - 1) / kSubpb2Threads); }

int subpb2_mesh_tables(long long n, long long n_el, const int* E, long long n_dir, const int* dir,
                       std::vector<int>& ptr, std::vector<int>& adj, std::vector<unsigned char>& kind, char* msg,
                       size_t msg_len) {
  std::vector<int> cnt((size_t)n + 1, 0), ids;
  ids.reserve((size_t)n_el * 8);
  for (long long e = 0; e < n_el; ++e)
    for (int k = 0; k < 8; ++k) {
      const int id = E[(size_t)e + (size_t)k * n_el];
      if (id < 0 || id > n || (k < 4 && id == 0)) {
        std::snprintf(msg, msg_len, "element %lld node %d: %d (corners 1..n, mid-side 0..n)", e + 1, k + 1, id);
        return 1;
      }
      ids.push_back(id);
      if (id) ++cnt[(size_t)id];
    }
  ptr.assign((size_t)n + 1, 0);
  for (long long i = 0; i < n; ++i) ptr[(size_t)i + 1] = ptr[(size_t)i] + cnt[(size_t)i + 1];
  adj.assign((size_t)ptr[(size_t)n], 0);
  std::vector<int> pos(ptr.begin(), ptr.end() - 1);
  for (long long e = 0; e < n_el; ++e)
    for (int k = 0; k < 8; ++k) {
      const int id = E[(size_t)e + (size_t)k * n_el];
      if (id) adj[(size_t)pos[(size_t)id - 1]++] = (int)(e * 8 + k);
    }
  // involved: unique(elementsFEM(:, 1:8)) less its first entry (:234-238: the reference
  // drops the 0 that absent mid-side nodes leave there); then the dirichlet nodes
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  kind.assign((size_t)n, 0);
  for (size_t k = 1; k < ids.size(); ++k) kind[(size_t)ids[k] - 1] = 1;
  for (long long k = 0; k < n_dir; ++k) {
    const int d = dir[k];
    if (d < 1 || d > n) {
      std::snprintf(msg, msg_len, "dirichlet node %d outside 1..%lld", d, n);
      return 1;
    }
    kind[(size_t)d - 1] = 2;
  }
  return 0;
}

size_t subpb2_scalars_bytes() { return sizeof(Subpb2Scalars); }

void subpb2_read_status(const void* host_copy, int* it, int* done, int* ok) {
  const Subpb2Scalars* s = (const Subpb2Scalars*)host_copy;
  *it = s->it;
  *done = s->done;
  *ok = s->ok;
}

int launch_subpb2_setup(int n_el, const int* elem, const double* coords, long long n, const double* U,
                        const double* F, int order, double beta, double mu, double alpha, const int* adj_ptr,
                        const int* adj, const unsigned char* free_, double* Ke, double* be, double* b, double* D,
                        double* x, double* r, double* z, double* p, double* part, Subpb2Scalars* sc,
                        cudaStream_t st) {
  const long long rows = 8LL * n_el;
  subpb2_element_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(n_el, elem, coords, n, U, F, order, beta, mu,
                                                                        alpha, Ke, be);
  const int nb = subpb2_blocks(n);
  subpb2_rhs_kernel<<<nb, kSubpb2Threads, 0, st>>>(n, adj_ptr, adj, Ke, be, free_, U, b, D, x);
  subpb2_start_kernel<<<nb, kSubpb2Threads, 0, st>>>(n, adj_ptr, adj, elem, n_el, Ke, free_, b, D, x, r, z, p, part);
  subpb2_init_scalars_kernel<<<1, kSubpb2Threads, 0, st>>>(part, nb, sc);
  return 4;
}

int launch_subpb2_iterations(int iters, int n_el, const int* elem, long long n, const int* adj_ptr, const int* adj,
                             const double* Ke, const unsigned char* free_, const double* D, double* x, double* r,
                             double* z, double* p, double* q, double* part, double tol2, int maxit,
                             Subpb2Scalars* sc, cudaStream_t st) {
  const int nb = subpb2_blocks(n);
  for (int k = 0; k < iters; ++k) {
    subpb2_matvec_kernel<<<nb, kSubpb2Threads, 0, st>>>(n, adj_ptr, adj, elem, n_el, Ke, free_, p, q, part, sc);
    subpb2_alpha_kernel<<<1, kSubpb2Threads, 0, st>>>(part, nb, sc);
    subpb2_update_kernel<<<nb, kSubpb2Threads, 0, st>>>(n, free_, D, p, q, x, r, z, part, sc);
    subpb2_beta_kernel<<<1, kSubpb2Threads, 0, st>>>(part, nb, tol2, maxit, sc);
    subpb2_direction_kernel<<<nb, kSubpb2Threads, 0, st>>>(n, free_, z, p, sc);
  }
  return 5 * iters;
}

}  // namespace aldic
