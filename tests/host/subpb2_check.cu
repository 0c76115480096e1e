// Host run of the global finite-element step (subpb2.cu): element rows from
// subpb2_element_row, the mesh tables from subpb2_mesh_tables, the right-hand side and the
// products from subpb2_gather_row, and the kernels' Jacobi-preconditioned CG steps in
// sequence.  Input file: int64 n, n_el, n_dir; int order; double beta, mu, alpha, tol;
// coords (2n, column-major), elements (8 n_el int32, column-major), U (2n), F (4n), dirichlet
// (n_dir int32).  Output file: K_e (64 n_el), b_e (16 n_el), Uhat (2n) doubles, then int32
// iterations, converged, kinds (n).
#include "../../3d-stereo-aldic_b200/csrc/subpb2.cu"

#include <cmath>
#include <cstdio>
#include <vector>

using namespace aldic;

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  long long hdr[3];
  int order;
  double par[4];
  if (std::fread(hdr, 8, 3, f) != 3 || std::fread(&order, 4, 1, f) != 1 || std::fread(par, 8, 4, f) != 4) return 4;
  const long long n = hdr[0], n_el = hdr[1], n_dir = hdr[2];
  std::vector<double> coords(2 * n), U(2 * n), F(4 * n);
  std::vector<int> E(8 * n_el), dir(n_dir > 0 ? n_dir : 1);
  if (std::fread(coords.data(), 8, 2 * n, f) != (size_t)(2 * n)) return 5;
  if (std::fread(E.data(), 4, 8 * n_el, f) != (size_t)(8 * n_el)) return 5;
  if (std::fread(U.data(), 8, 2 * n, f) != (size_t)(2 * n)) return 5;
  if (std::fread(F.data(), 8, 4 * n, f) != (size_t)(4 * n)) return 5;
  if (n_dir > 0 && std::fread(dir.data(), 4, n_dir, f) != (size_t)n_dir) return 5;
  std::fclose(f);
  const double beta = par[0], mu = par[1], alpha = par[2], tol = par[3];

  // element rows, as subpb2_element_kernel computes them
  std::vector<double> Ke(64 * n_el, 0.0), be(16 * n_el, 0.0);
  for (long long e = 0; e < n_el; ++e) {
    int id[8];
    for (int k = 0; k < 8; ++k) id[k] = E[e + k * n_el];
    double xy[16], ue[16], d[4];
    for (int k = 0; k < 8; ++k) {
      const bool on = id[k] != 0;
      const long long g = id[k] - 1;
      xy[2 * k] = on ? coords[g] : 0.0;
      xy[2 * k + 1] = on ? coords[g + n] : 0.0;
      ue[2 * k] = on ? U[2 * g] : 0.0;
      ue[2 * k + 1] = on ? U[2 * g + 1] : 0.0;
    }
    for (int k = 0; k < 4; ++k) d[k] = id[4 + k] != 0 ? 1.0 : 0.0;
    for (int a = 0; a < 8; ++a) {
      if (id[a] == 0) continue;
      double fa[4];
      for (int k = 0; k < 4; ++k) fa[k] = F[4 * (id[a] - 1) + k];
      subpb2_element_row(a, xy, d, ue, fa, order, beta, mu, alpha, &Ke[64 * e + 8 * a], &be[16 * e + 2 * a]);
    }
  }
  std::vector<int> ptr, adj;
  std::vector<unsigned char> kind;
  char msg[160];
  if (subpb2_mesh_tables(n, n_el, E.data(), n_dir, dir.data(), ptr, adj, kind, msg, sizeof(msg))) {
    std::printf("%s\n", msg);
    return 6;
  }
  // the kernels' steps
  std::vector<double> b(2 * n), D(n), x(2 * n), r(2 * n, 0.0), z(2 * n, 0.0), p(2 * n, 0.0), q(2 * n, 0.0);
  for (long long i = 0; i < n; ++i) {
    double bx = 0, by = 0, dg = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
      const int e = adj[k] >> 3, s = adj[k] & 7;
      bx += be[16 * e + 2 * s];
      by += be[16 * e + 2 * s + 1];
      dg += Ke[64 * e + 9 * s];
    }
    b[2 * i] = bx;
    b[2 * i + 1] = by;
    D[i] = dg;
    x[2 * i] = kind[i] == 2 ? U[2 * i] : 0.0;
    x[2 * i + 1] = kind[i] == 2 ? U[2 * i + 1] : 0.0;
  }
  double rz = 0, rr0 = 0;
  for (long long i = 0; i < n; ++i) {
    if (kind[i] != 1) continue;
    double kx, ky;
    subpb2_gather_row(i, ptr.data(), adj.data(), E.data(), (int)n_el, Ke.data(), x.data(), kx, ky);
    r[2 * i] = b[2 * i] - kx;
    r[2 * i + 1] = b[2 * i + 1] - ky;
    for (int c = 0; c < 2; ++c) {
      z[2 * i + c] = r[2 * i + c] / D[i];
      p[2 * i + c] = z[2 * i + c];
      rz += r[2 * i + c] * z[2 * i + c];
      rr0 += r[2 * i + c] * r[2 * i + c];
    }
  }
  int it = 0, ok = 1;
  bool done = rr0 == 0.0;
  const int maxit = (int)std::min<long long>(20 * n + 1000, 200000);
  while (!done) {
    double pq = 0;
    for (long long i = 0; i < n; ++i) {
      double qx = 0, qy = 0;
      if (kind[i] == 1) subpb2_gather_row(i, ptr.data(), adj.data(), E.data(), (int)n_el, Ke.data(), p.data(), qx, qy);
      q[2 * i] = qx;
      q[2 * i + 1] = qy;
      pq += p[2 * i] * qx + p[2 * i + 1] * qy;
    }
    if (!(pq > 0)) {
      ok = 0;
      break;
    }
    const double al = rz / pq;
    double rzn = 0, rr = 0;
    for (long long i = 0; i < n; ++i) {
      if (kind[i] != 1) continue;
      for (int c = 0; c < 2; ++c) {
        const long long k = 2 * i + c;
        x[k] += al * p[k];
        r[k] -= al * q[k];
        z[k] = r[k] / D[i];
        rzn += r[k] * z[k];
        rr += r[k] * r[k];
      }
    }
    const double bt = rzn / rz;
    rz = rzn;
    ++it;
    if (rr <= tol * tol * rr0 || it >= maxit) {
      done = true;
      if (rr > tol * tol * rr0) ok = 0;
    }
    for (long long i = 0; i < n; ++i)
      if (kind[i] == 1)
        for (int c = 0; c < 2; ++c) p[2 * i + c] = z[2 * i + c] + bt * p[2 * i + c];
  }
  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 7;
  std::fwrite(Ke.data(), 8, Ke.size(), o);
  std::fwrite(be.data(), 8, be.size(), o);
  std::fwrite(x.data(), 8, x.size(), o);
  int st[2] = {it, ok};
  std::fwrite(st, 4, 2, o);
  std::vector<int> kd(kind.begin(), kind.end());
  std::fwrite(kd.data(), 4, kd.size(), o);
  std::fclose(o);
  std::printf("iterations %d converged %d\n", it, ok);
  return 0;
}
