// Host-side check of the tcgen05 pair kernel's shared-memory layout
// (alglin_b200/csrc/bcr_umma.cuh, umma_layout / umma_fits) for every shape the
// kernel accepts: the regions that are live at the same time do not overlap,
// every operand address is 16-byte aligned, the K-major operand tiles stay
// inside their regions, and the total fits one CTA's shared memory.
#include <cstdint>
#include <cstdio>

#include "bcr_common.cuh"

namespace bcr {
#include "bcr_umma_layout.cuh"
}

int main() {
  using namespace bcr;
  int checked = 0, failures = 0;
  for (int n = 33; n <= UM_NMAX; ++n)
    for (int nr = 0; nr <= UM_NRMAX; ++nr)
      for (int nx = 0; nx <= UM_NXMAX; ++nx) {
        Dims d{};
        d.nblock = 8; d.n = n; d.nr = nr; d.nx = nx;
        if (!umma_fits(d)) { std::printf("not accepted: n=%d nr=%d nx=%d\n", n, nr, nx); ++failures; continue; }
        const UmmaLayout L = umma_layout(d);
        const unsigned endA = 2u * L.szAhalf, endB = L.offB + 4u * L.szBhalf;
        const unsigned endP = (unsigned)(L.R * L.LDP * 4), endZ = L.offZ + (unsigned)(L.NP * L.LDP * 4);
        const unsigned endLc = L.offLc + (unsigned)(UM_NRMAX * n * 4);
        bool ok = true;
        ok &= L.offB == endA;                           // B buffers after the A operand
        ok &= L.offZ >= endA && L.offZ >= endP;         // Z is read while A is written; P is read while Z is written
        ok &= L.offLc >= endB && L.offLc >= endZ;       // Lc is read while the B buffers are written
        ok &= L.bytes >= endB && L.bytes >= endLc;
        ok &= L.bytes + 4096 <= 227u * 1024u;            // with the static shared memory
        ok &= (L.offB % 16) == 0 && (L.szAhalf % 16) == 0 && (L.szBhalf % 16) == 0 && (L.offZ % 16) == 0;
        ok &= (L.LBO_B % 16) == 0 && (L.LBO_B / 4) % 32 == 8 && L.LBO_B >= L.Npad * 16;
        ok &= L.Kpad % 16 == 0 && L.Kpad >= n && L.Npad % 16 == 0 && L.Npad >= 2 * n + nx;
        ok &= L.N0 % 16 == 0 && L.N1 % 16 == 0 && L.N0 + L.N1 == L.Npad && L.N0 <= 256 && L.N1 <= 256;
        ok &= 16 * L.Npad <= UM_PF * UM_NT && L.R <= UM_NT;
        ok &= L.LDP % 4 == 0 && (L.LDP / 4) % 2 == 1 && L.LDP >= L.NP + 4;
        // the trailing rows by position fit the CTA's slab of the CTA-per-pair kernels
        ok &= (long)2 * n * (2 * n + nx) <= (long)(2 * n + nr) * (3 * n + nx);
        // the last A and B tile elements lie inside their halves
        ok &= (unsigned)((L.Kpad / 4 - 1) * 2048 + 15 * 128 + 7 * 16 + 12 + 4) <= L.szAhalf;
        ok &= (unsigned)(3 * L.LBO_B + (L.Npad / 8 - 1) * 128 + 7 * 16 + 12 + 4) <= L.szBhalf;
        if (!ok) {
          std::printf("layout check failed: n=%d nr=%d nx=%d\n", n, nr, nx);
          ++failures;
        }
        ++checked;
      }
  std::printf("%d shapes checked, %d failures\n", checked, failures);
  return failures ? 1 : 0;
}
