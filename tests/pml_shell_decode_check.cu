// Host-side check of the PML shell decoder and its multiply-shift division
// (tlm_kernels.cuh), built by tests/test_pml_shell_decode.py with nvcc and
// run on the CPU: no CUDA call is made.
//  1. fast_div(n, make_fast_div(d)) == n / d for divisors and dividends at
//     the edges (1, powers of two and their neighbours, 2^31 - 1) and random.
//  2. pml_shell_pos(s) reproduces the s-th PML cell of a brute-force
//     traversal (z outer, then y, then x) for random meshes and per-face
//     thicknesses, including faces without PML.
#include <cstdio>
#include <cstdint>
#include <random>
#include <vector>

#include "../ggi_tlm_b200/csrc/tlm_kernels.cuh"

static int check_div(std::mt19937_64 &rng) {
  std::vector<long long> ds = {1, 2, 3, 5, 7, 10, 255, 256, 257, 65535, 65536, 65537, 1000003, 2147483647LL};
  for (int k = 1; k < 31; k++) {
    ds.push_back((1LL << k) - 1);
    ds.push_back(1LL << k);
    ds.push_back((1LL << k) + 1);
  }
  for (int i = 0; i < 2000; i++) ds.push_back((long long)(rng() % 2147483647ULL) + 1);
  for (int i = 0; i < 2000; i++) ds.push_back((long long)(rng() % 100000ULL) + 1);
  long long bad = 0;
  for (long long d : ds) {
    if (d > 2147483647LL) continue;
    const tlm::FastDiv f = tlm::make_fast_div((int)d);
    std::vector<long long> ns = {0, 1, d - 1, d, d + 1, 2 * d - 1, 2 * d, 2147483647LL, 2147483646LL,
                                 2147483647LL - 2147483647LL % d, 2147483647LL - 2147483647LL % d - 1};
    for (int i = 0; i < 300; i++) ns.push_back((long long)(rng() % 2147483648ULL));
    for (int i = 0; i < 100; i++) {
      const long long q = (long long)(rng() % (2147483648ULL / (unsigned long long)d));
      ns.push_back(q * d);
      ns.push_back(q * d + d - 1);
    }
    for (long long n : ns) {
      if (n < 0 || n > 2147483647LL) continue;
      if (tlm::fast_div((int)n, f) != (int)(n / d)) {
        if (bad < 5) std::printf("fast_div(%lld, %lld) = %d, want %lld\n", n, d, tlm::fast_div((int)n, f), n / d);
        bad++;
      }
    }
  }
  return bad == 0;
}

static int check_shell(std::mt19937_64 &rng) {
  long long bad = 0;
  for (int trial = 0; trial < 400; trial++) {
    const int nx = 1 + (int)(rng() % 40), ny = 1 + (int)(rng() % 40), nz = 1 + (int)(rng() % 40);
    int t[6];
    for (int k = 0; k < 6; k++) t[k] = (int)(rng() % 7);  // 0: a face without PML
    const int xl = std::min(t[0], nx), xh = std::min(t[1], nx - xl);
    const int yl = std::min(t[2], ny), yh = std::min(t[3], ny - yl);
    const int zl = std::min(t[4], nz), zh = std::min(t[5], nz - zl);
    std::vector<int> px, py, pz;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++)
        for (int x = 0; x < nx; x++) {
          const bool in = z < zl || z >= nz - zh || y < yl || y >= ny - yh || x < xl || x >= nx - xh;
          if (in) { px.push_back(x); py.push_back(y); pz.push_back(z); }
        }
    tlm::PmlShell h{};
    h.on = 1;
    h.nx = nx; h.ny = ny; h.nz = nz;
    h.xl = xl; h.xh = xh; h.yl = yl; h.yh = yh; h.zl = zl; h.zh = zh;
    h.full = nx * ny;
    h.partial = (yl + yh) * nx + (ny - yl - yh) * (xl + xh);
    h.d_full = tlm::make_fast_div(h.full);
    h.d_nx = tlm::make_fast_div(nx);
    h.d_partial = tlm::make_fast_div(h.partial);
    h.d_w = tlm::make_fast_div(xl + xh);
    const long long count = (long long)(zl + zh) * h.full + (long long)(nz - zl - zh) * h.partial;
    if (count != (long long)px.size()) {
      if (bad < 5) std::printf("count %lld != %zu\n", count, px.size());
      bad++;
      continue;
    }
    for (size_t s = 0; s < px.size(); s++) {
      int x, y, z;
      tlm::pml_shell_pos(h, (int)s, x, y, z);
      if (x != px[s] || y != py[s] || z != pz[s]) {
        if (bad < 5)
          std::printf("mesh %dx%dx%d t=(%d,%d,%d,%d,%d,%d) cell %zu: (%d,%d,%d), want (%d,%d,%d)\n", nx, ny, nz, xl, xh,
                      yl, yh, zl, zh, s, x, y, z, px[s], py[s], pz[s]);
        bad++;
      }
    }
  }
  return bad == 0;
}

int main() {
  std::mt19937_64 rng(12345);
  const int a = check_div(rng), b = check_shell(rng);
  std::printf("fast_div %s, shell %s\n", a ? "ok" : "FAILED", b ? "ok" : "FAILED");
  return (a && b) ? 0 : 1;
}
