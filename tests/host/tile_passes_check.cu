// Host check of the shared-product algebra of the tile search (search_tile.cu): pass 1
// (row-band sums per tile row) followed by pass 2 (block sums over rows) must give, for
// every subset of a tile and every shift column, the window sum of f(x) g(x + d) over the
// (w+1)^2 window -- the numerator normxcorr2 forms per subset.  Random data, FP64 direct
// sums as the reference; run on the CPU through the functions' host forms.
#include "../../3d-stereo-aldic_b200/csrc/search_tile.cu"

#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

using namespace aldic;

template <int ST, int W1, int TI, int DBC>
int check_shape() {
  using S = TileShape<ST, W1, TI, DBC>;
  constexpr int FR = S::FR, FC = S::FC, FCP = S::FCP, GCP = S::GCP, FRP = S::FRP, H0 = S::H0;
  std::mt19937 rng(7 + ST * 100 + W1);
  std::uniform_real_distribution<float> U(-1.f, 1.f);
  std::vector<float> F(FR * FCP + 16, 0.f), G(FR * GCP + 16, 0.f), RB(kTJ * DBC * FRP + 16, 0.f);
  for (int x = 0; x < FR; ++x)
    for (int c = 0; c < FCP; ++c) F[x * FCP + c] = c < FC ? U(rng) : 0.f;
  for (int x = 0; x < FR; ++x)
    for (int c = 0; c < GCP; ++c) G[x * GCP + c] = c < FC + DBC - 1 ? U(rng) : 0.f;
  // pass 1: every tile row, every group of 8 shift columns
  for (int grp = 0; grp < DBC / 8; ++grp)
    for (int x = 0; x < FR; ++x) {
      if constexpr (ST % 2 == 0)
        row_band_sums_x2<ST, W1, FC, FRP, DBC>(&F[x * FCP], &G[x * GCP] + grp * 8, &RB[(grp * 8) * FRP + x]);
      else
        row_band_sums<ST, W1, FC, FRP, DBC>(&F[x * FCP], &G[x * GCP] + grp * 8, &RB[(grp * 8) * FRP + x]);
    }
  int bad = 0;
  double worst = 0.0;
  for (int j = 0; j < kTJ; ++j)
    for (int d = 0; d < DBC; ++d) {
      const float* rb = &RB[(j * DBC + d) * FRP];
      float N[TI];
      {
        float N0[H0];
        if constexpr (ST % 2 == 0)
          column_sums_x2<ST, W1, H0, 0>(rb, N0);
        else
          column_sums<ST, W1, H0, 0>(rb, N0);
        for (int e = 0; e < H0; ++e) N[e] = N0[e];
      }
      if constexpr (TI - H0 > 0) {
        float N1[TI - H0];
        if constexpr (ST % 2 == 0)
          column_sums_x2<ST, W1, TI - H0, H0 * ST>(rb, N1);
        else
          column_sums<ST, W1, TI - H0, H0 * ST>(rb, N1);
        for (int e = 0; e < TI - H0; ++e) N[H0 + e] = N1[e];
      }
      for (int i = 0; i < TI; ++i) {
        double ref = 0.0, mag = 0.0;
        for (int a = 0; a < W1; ++a)
          for (int b = 0; b < W1; ++b) {
            const double p = (double)F[(i * ST + a) * FCP + j * ST + b] * G[(i * ST + a) * GCP + j * ST + b + d];
            ref += p;
            mag += std::fabs(p);
          }
        const double err = std::fabs(N[i] - ref) / (mag > 0 ? mag : 1.0);
        worst = err > worst ? err : worst;
        if (err > 1e-5) {
          if (bad < 5) std::printf("ST %d W1 %d: subset (%d, %d) shift %d: %g vs %g\n", ST, W1, i, j, d, N[i], ref);
          ++bad;
        }
      }
    }
  std::printf("ST %d W1 %d TI %d DBC %d: %d of %d window sums off (worst relative %.2e)\n", ST, W1, TI, DBC, bad,
              kTJ * DBC * TI, worst);
  return bad;
}

int main() {
  int bad = 0;
  bad += check_shape<10, 41, TileFor<10, 41, 24>::TI, 24>();
  bad += check_shape<10, 41, TileFor<10, 41, 16>::TI, 16>();
  bad += check_shape<16, 31, TileFor<16, 31, 16>::TI, 16>();
  bad += check_shape<16, 33, TileFor<16, 33, 16>::TI, 16>();
  bad += check_shape<12, 21, TileFor<12, 21, 16>::TI, 16>();
  bad += check_shape<9, 17, TileFor<9, 17, 16>::TI, 16>();
  bad += check_shape<8, 33, TileFor<8, 33, 16>::TI, 16>();
  return bad ? 1 : 0;
}
