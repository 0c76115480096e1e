// Host run of the bad-point removal's per-entry algebra (outliers.cu): the method-3
// operator's coefficients, a sequential CGLS that takes the same steps as
// inpaint_del4_kernel, and the single-precision median test, through the functions' host
// forms.  Input file: int m, n; then A (with NaN), X0 (warm start), U, V (filled grids),
// mn doubles each.  Output file: coefficients (mn x 13 doubles), the method-3 fill of A
// (mn doubles), the kept-row flags (mn ints), |normalised fluctuation| (mn floats).
#include "../../3d-stereo-aldic_b200/csrc/outliers.cu"

#include <cstdio>
#include <vector>

using namespace aldic;

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  int m = 0, n = 0;
  if (std::fread(&m, 4, 1, f) != 1 || std::fread(&n, 4, 1, f) != 1) return 4;
  const int mn = m * n;
  std::vector<double> A(mn), X0(mn), U(mn), V(mn);
  for (auto* v : {&A, &X0, &U, &V})
    if (std::fread(v->data(), 8, mn, f) != (size_t)mn) return 5;
  std::fclose(f);

  std::vector<double> coef((size_t)mn * 13);
  for (int g = 0; g < mn; ++g)
    for (int o = 0; o < 13; ++o) {
      int dr, dc;
      del4_tap(o, dr, dc);
      coef[(size_t)g * 13 + o] = del4_coef(g % m, g / m, m, n, dr, dc);
    }

  // CGLS, the kernel's steps in sequence
  std::vector<int> map(mn, -1), emap(mn, -1), list, elist, eqflag(mn, 0);
  for (int g = 0; g < mn; ++g)
    if (A[g] != A[g]) {
      map[g] = (int)list.size();
      list.push_back(g);
    }
  for (int g = 0; g < mn; ++g)
    if (del4_touches_nan(g, m, n, A.data())) {
      emap[g] = (int)elist.size();
      elist.push_back(g);
      eqflag[g] = 1;
    }
  const int nu = (int)list.size(), ne = (int)elist.size();
  std::vector<double> x(nu), s(nu), p(nu), rv(ne), q(ne), out(A);
  int it = 0;
  bool met = true;
  if (nu > 0) {
    for (int t = 0; t < ne; ++t) rv[t] = del4_rhs(elist[t], m, n, A.data());
    for (int u = 0; u < nu; ++u) x[u] = X0[list[u]];
    double atb = 0.0;
    for (int u = 0; u < nu; ++u) {
      const double v = del4_col(list[u], m, n, emap.data(), rv.data());
      atb += v * v;
    }
    for (int t = 0; t < ne; ++t) rv[t] -= del4_row(elist[t], m, n, map.data(), x.data());
    double gamma = 0.0;
    for (int u = 0; u < nu; ++u) {
      s[u] = p[u] = del4_col(list[u], m, n, emap.data(), rv.data());
      gamma += s[u] * s[u];
    }
    const double target = 1e-24 * atb;
    const int maxit = 8 * mn + 200 < 20000 ? 8 * mn + 200 : 20000;
    met = gamma <= target;
    while (!met && it < maxit) {
      double qq = 0.0;
      for (int t = 0; t < ne; ++t) {
        q[t] = del4_row(elist[t], m, n, map.data(), p.data());
        qq += q[t] * q[t];
      }
      if (!(qq > 0.0)) break;
      const double alpha = gamma / qq;
      for (int u = 0; u < nu; ++u) x[u] += alpha * p[u];
      for (int t = 0; t < ne; ++t) rv[t] -= alpha * q[t];
      double gn = 0.0;
      for (int u = 0; u < nu; ++u) {
        s[u] = del4_col(list[u], m, n, emap.data(), rv.data());
        gn += s[u] * s[u];
      }
      ++it;
      met = gn <= target;
      const double beta = gn / gamma;
      gamma = gn;
      for (int u = 0; u < nu; ++u) p[u] = s[u] + beta * p[u];
    }
    for (int u = 0; u < nu; ++u) out[list[u]] = x[u];
  }

  std::vector<float> fu(mn), fv(mn), mag(mn);
  for (int g = 0; g < mn; ++g) {
    fu[g] = med_fluct(U.data(), m, n, g % m, g / m);
    fv[g] = med_fluct(V.data(), m, n, g % m, g / m);
  }
  for (int g = 0; g < mn; ++g) mag[g] = norm_fluct_mag(fu.data(), fv.data(), m, n, g % m, g / m);

  FILE* o = std::fopen(argv[2], "wb");
  if (!o) return 6;
  std::fwrite(coef.data(), 8, coef.size(), o);
  std::fwrite(out.data(), 8, mn, o);
  std::fwrite(eqflag.data(), 4, mn, o);
  std::fwrite(mag.data(), 4, mn, o);
  std::fclose(o);
  std::printf("unknowns %d rows %d iterations %d met %d\n", nu, ne, it, met ? 1 : 0);
  return 0;
}
