// schema_driver.cpp -- C++ caller of libdicegpu.so through include/dicegpu.hpp.
//
// Like the reference's component-test executables it prints "TEST PASSED"
// on success (tests/CMakeLists.txt:11-18).  A speckle pattern of Gaussian
// blobs is evaluated analytically at x and at x - (u, v), so the deformed
// image is exact (no resampling); every subset must recover (u, v) within
// 0.01 px with the reference's status flag 1.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "dicegpu.hpp"

namespace {
struct Blob {
  double x, y, s, a;
};

std::vector<float> render(int w, int h, const std::vector<Blob>& blobs, double du, double dv) {
  std::vector<float> img((size_t)w * h, 20.0f);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      double v = 20.0;
      for (const Blob& b : blobs) {
        const double dx = x - du - b.x, dy = y - dv - b.y;
        const double d2 = dx * dx + dy * dy;
        if (d2 < 36.0 * b.s * b.s) v += b.a * std::exp(-d2 / (2.0 * b.s * b.s));
      }
      img[(size_t)y * w + x] = (float)v;
    }
  return img;
}
}  // namespace

int main() {
  const int w = 160, h = 120;
  const double u = 0.37, v = -1.21;
  std::mt19937 rng(7);
  std::uniform_real_distribution<double> ux(-5.0, w + 5.0), uy(-5.0, h + 5.0), us(1.2, 2.2), ua(60.0, 180.0);
  std::vector<Blob> blobs(900);
  for (Blob& b : blobs) b = Blob{ux(rng), uy(rng), us(rng), ua(rng)};
  const std::vector<float> ref = render(w, h, blobs, 0.0, 0.0);
  const std::vector<float> def = render(w, h, blobs, u, v);

  dicegpu_params p = dicegpu::default_params();
  p.subset_size = 21;
  p.enable_rotation = 1;
  p.fast_solver_tolerance = 1e-5;
  int failures = 0;
  try {
    dicegpu::Schema schema(p);
    schema.set_ref_image(w, h, ref.data());
    std::vector<double> cx, cy;
    for (int y = 30; y <= h - 30; y += 15)
      for (int x = 30; x <= w - 30; x += 15) {
        cx.push_back(x);
        cy.push_back(y);
      }
    schema.set_subsets(cx, cy);
    schema.set_def_image(w, h, def.data());
    if (schema.execute_correlation() != 0) ++failures;
    for (int i = 0; i < schema.num_subsets(); ++i) {
      const double gu = schema.global_field_value(i, DICEGPU_F_DISP_X);
      const double gv = schema.global_field_value(i, DICEGPU_F_DISP_Y);
      const double st = schema.global_field_value(i, DICEGPU_F_STATUS);
      if (std::fabs(gu - u) > 0.01 || std::fabs(gv - v) > 0.01 || st != 1.0) {
        std::printf("subset %d at (%g,%g): u %.5f v %.5f status %g\n", i, cx[i], cy[i], gu, gv, st);
        ++failures;
      }
    }
    std::printf("%d subsets correlated\n", schema.num_subsets());
    // the ABI's argument checks surface as exceptions on the C++ side
    bool threw = false;
    try {
      schema.global_field_value(schema.num_subsets(), 0);
    } catch (const dicegpu::Error&) {
      threw = true;
    }
    if (!threw) ++failures;
  } catch (const dicegpu::Error& e) {
    std::printf("error: %s\n", e.what());
    ++failures;
  }
  if (failures) {
    std::printf("TEST FAILED (%d)\n", failures);
    return 1;
  }
  std::printf("TEST PASSED\n");
  return 0;
}
