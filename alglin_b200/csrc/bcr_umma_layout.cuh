// Shared-memory and slab layout of the tcgen05 pair kernel (bcr_umma.cuh) and
// the shapes it accepts; included inside namespace bcr.
#pragma once

constexpr int UM_NT = 384;              // threads per CTA
constexpr int UM_NW = UM_NT / 32;
constexpr int UM_NMAX = 128, UM_NRMAX = 16, UM_NXMAX = 16;
constexpr int UM_TMEM_COLS = 512;
constexpr int UM_BW = 16;  // panel column block of the LU (registers per row)
constexpr int UM_PF = 12;  // B-operand elements per thread and stage: 16 * (2n + nx) <= UM_PF * UM_NT

struct UmmaLayout {
  int R, NP, LDP, Kpad, Nc, Npad, N0, N1, LBO_B;
  unsigned szAhalf, offB, szBhalf, offZ, offLc, bytes;
};

__host__ __device__ inline UmmaLayout umma_layout(const Dims& d) {
  UmmaLayout L;
  const int n = d.n;
  L.R = 2 * n + d.nr;
  L.NP = (n + 31) / 32 * 32;
  L.LDP = L.NP + 4;  // rows 16-byte aligned, 8 consecutive rows on distinct banks
  L.Kpad = (n + 15) / 16 * 16;
  L.Nc = 2 * n + d.nx;
  L.Npad = (L.Nc + 15) / 16 * 16;
  if (L.Npad <= 256) { L.N0 = L.Npad; L.N1 = 0; }
  else { L.N0 = (L.Npad / 2 + 15) / 16 * 16; L.N1 = L.Npad - L.N0; }
  int lbo = L.Npad * 16;
  while ((lbo / 4) % 32 != 8) lbo += 16;  // the 4 K groups of a stage on distinct banks
  L.LBO_B = lbo;
  L.szAhalf = (unsigned)(L.Kpad / 4) * 2048u;      // 128 rows x Kpad, one of hi / lo
  L.offB = 2 * L.szAhalf;
  L.szBhalf = 4u * (unsigned)lbo;                  // Npad rows x 16, one of hi / lo
  const unsigned endB = L.offB + 4 * L.szBhalf;    // two stages of (hi, lo)
  // Z is read while the A operand is written, and Lc is read between the two
  // products: neither may overlap the operand regions
  L.offZ = ((unsigned)(L.R * L.LDP * 4) + 15u) & ~15u;
  if (L.offZ < L.offB) L.offZ = L.offB;
  L.offLc = L.offZ + (unsigned)(L.NP * L.LDP * 4);
  if (L.offLc < endB) L.offLc = endB;
  const unsigned endS = L.offLc + (unsigned)(UM_NRMAX * n * 4);
  L.bytes = endB > endS ? endB : endS;
  return L;
}

__host__ inline bool umma_fits(const Dims& d) {
  return d.n > 32 && d.n <= UM_NMAX && d.nr <= UM_NRMAX && d.nx <= UM_NXMAX &&
         16 * umma_layout(d).Npad <= UM_PF * UM_NT &&
         umma_layout(d).bytes + 4096 <= 227u * 1024u;  // with the static shared memory
}
