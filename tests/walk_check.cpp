// Host check of the exact path walks in doi_b200/csrc/rte_walk.cuh (compiled by g++ from
// tests/test_walk_cpu.py): on random grids, voxel pairs and fields,
//  (1) path_sum<float> (crossing parameters carried in FP32) equals, bit for bit, the same walk with
//      integer crossing parameters written out below;
//  (2) path_sum_box over a field that is zero outside a random box equals path_sum bit for bit, in FP32
//      and FP64 sums.
// Prints "pairs <n> nonzero <n> mismatches <n>" and exits 1 on any mismatch.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "rte_walk.cuh"

// the integer-parameter form of the walk (FP32 sum): crossings compared as integers, the segment
// length converted to FP32 at every step
static float walk_int(int i, int j, int k, int ip, int jp, int kp, const double* mu, int nx, int plane) {
  const int Dz = std::abs(ip - i), Dy = std::abs(jp - j), Dx = std::abs(kp - k);
  const int mz = Dz > 1 ? Dz : 1, my = Dy > 1 ? Dy : 1, mx = Dx > 1 ? Dx : 1;
  const int Q = 2 * mx * my * mz, BIG = 0x3fffffff;
  const int incz = 2 * mx * my, incy = 2 * mx * mz, incx = 2 * my * mz;
  int Az = Dz ? mx * my : BIG, Ay = Dy ? mx * mz : BIG, Ax = Dx ? my * mz : BIG;
  const int stz = ip > i ? plane : -plane, sty = jp > j ? nx : -nx, stx = kp > k ? 1 : -1;
  int v = i * plane + j * nx + k, prev = 0;
  float acc = 0.f;
  for (int s = 0; s < Dx + Dy + Dz; ++s) {
    const int m = std::min(Az, std::min(Ay, Ax));
    acc = std::fma((float)mu[v], (float)(m - prev), acc);
    prev = m;
    const bool bz = Az == m, by = !bz && Ay == m, bx = !bz && !by;
    v += bz ? stz : (by ? sty : stx);
    Az += bz ? incz : 0;
    Ay += by ? incy : 0;
    Ax += bx ? incx : 0;
  }
  return std::fma((float)mu[v], (float)(Q - prev), acc);
}

template <typename T>
static bool same(T a, T b) { return std::memcmp(&a, &b, sizeof(T)) == 0; }

int main() {
  std::mt19937 rng(12345);
  std::uniform_real_distribution<double> U(-1.0, 2.0);
  long pairs = 0, nonzero = 0, bad = 0;
  for (int t = 0; t < 4000; ++t) {
    const int nx = 2 + rng() % 40, ny = 2 + rng() % 40, nz = 2 + rng() % 40, plane = nx * ny;
    const int dim[3] = {nx, ny, nz};
    int lo[3], hi[3];
    for (int q = 0; q < 3; ++q) {
      const int a = rng() % dim[q], b = rng() % dim[q];
      lo[q] = std::min(a, b);
      hi[q] = std::max(a, b);
    }
    std::vector<double> full((size_t)nx * ny * nz), box((size_t)nx * ny * nz, 0.0);
    for (auto& x : full) x = U(rng);
    for (int z = lo[2]; z <= hi[2]; ++z)
      for (int y = lo[1]; y <= hi[1]; ++y)
        for (int x = lo[0]; x <= hi[0]; ++x)
          if (rng() % 4) box[(size_t)z * plane + y * nx + x] = U(rng);
    for (int p = 0; p < 50; ++p, ++pairs) {
      const int i = rng() % nz, j = rng() % ny, k = rng() % nx;
      const int ip = rng() % nz, jp = rng() % ny, kp = rng() % nx;
      int Q1, Q2, Q3;
      const float a = path_sum<float, double>(i, j, k, ip, jp, kp, full.data(), nx, plane, Q1);
      if (!same(a, walk_int(i, j, k, ip, jp, kp, full.data(), nx, plane))) ++bad;
      const float bf = path_sum<float, double>(i, j, k, ip, jp, kp, box.data(), nx, plane, Q1);
      const float cf = path_sum_box<float, double>(i, j, k, ip, jp, kp, box.data(), nx, plane, lo, hi, Q2);
      const double bd = path_sum<double, double>(i, j, k, ip, jp, kp, box.data(), nx, plane, Q1);
      const double cd = path_sum_box<double, double>(i, j, k, ip, jp, kp, box.data(), nx, plane, lo, hi, Q3);
      if (!same(bf, cf) || !same(bd, cd) || Q1 != Q2 || Q1 != Q3) ++bad;
      if (bf != 0.f) ++nonzero;
    }
  }
  std::printf("pairs %ld nonzero %ld mismatches %ld\n", pairs, nonzero, bad);
  return bad ? 1 : 0;
}
