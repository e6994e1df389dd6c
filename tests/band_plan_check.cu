// Host-only check of the staging plan of the bulk-copy band products
// (tnl_b200/csrc/band.cuh): for random ascending diagonal offsets with 6 to
// 8 diagonals, including 0, within the +-32767 the diagonal copies allow,
// and for the operand sets the library plans, every bulk copy
// band_issue would issue has a 16-byte-aligned shared-memory destination,
// global source and size; each band run fits the stage slot planned for it
// and covers every in-range column of the tile's rows; the interior-tile
// offsets (xoff, selfoff) agree with the run starts; and the stages fit the
// shared memory of one block.  Prints one line "ok <cases>" or the first
// violation, and returns non-zero on a violation.
#include <cstdint>
#include <cstdio>
#include <random>

#include "band.cuh"

using namespace tnlb;

namespace {

// band_start of the device code, on the host
int64_t run_start(int32_t lo, int64_t i0)
{
   const int64_t s = (i0 + lo) & ~(int64_t)3;
   return s < 0 ? 0 : s;
}

int fail(const char* what, int D, const int32_t* o, int64_t n, int64_t i0)
{
   std::printf("violation: %s (D=%d, n=%lld, i0=%lld, offsets", what, D, (long long)n, (long long)i0);
   for (int j = 0; j < D; j++) std::printf(" %d", o[j]);
   std::printf(")\n");
   return 1;
}

struct Operands {
   int vbytes, KB, KO, KD;
};

}  // namespace

int main()
{
   // the operand sets planned by the library: the FP16 factor product with
   // two banded inputs (k_band_g_update), the FP16 transposed factor with
   // one banded input and own FP32 and FP64 rows (k_band_gt_xpby), and the
   // FP32 operator copy with one banded input (compact_band_capable)
   const Operands sets[] = {{2, 2, 0, 0}, {2, 1, 1, 1}, {4, 1, 0, 0}};
   const int64_t sizes[] = {1, 3, 1023, 1024, 1025, 4097, 70000, 262147};
   std::mt19937 rng(12345);
   long cases = 0;
   for (int trial = 0; trial < 4000; trial++) {
      const int D = 6 + (int)(rng() % 3);
      // ascending offsets with 0 among them: some clustered within the band
      // gap, some far apart
      int32_t o[8];
      const int zero_at = (int)(rng() % D);
      o[zero_at] = 0;
      for (int j = zero_at - 1; j >= 0; j--) {
         const int32_t step = rng() % 2 ? 1 + (int32_t)(rng() % 20) : 1 + (int32_t)(rng() % 4000);
         o[j] = o[j + 1] - step;
      }
      for (int j = zero_at + 1; j < D; j++) {
         const int32_t step = rng() % 2 ? 1 + (int32_t)(rng() % 20) : 1 + (int32_t)(rng() % 4000);
         o[j] = o[j - 1] + step;
      }
      if (o[0] < -32767 || o[D - 1] > 32767) continue;
      for (const Operands& ops : sets) {
         const BandPlan P = band_plan(o, D, ops.vbytes, ops.KB, ops.KO, ops.KD);
         if (P.stages < 2 || P.stages > kBandStages) return fail("stage count", D, o, 0, 0);
         // one block's dynamic shared memory, beside its static barriers
         if ((size_t)P.stages * P.bytes > 227 * 1024 - 1024) return fail("stages exceed a block", D, o, 0, 0);
         if (P.bytes % 128 || P.vals % 128) return fail("stage alignment", D, o, 0, 0);
         for (int k = 0; k < ops.KB; k++)
            for (int b = 0; b < P.nb; b++)
               if (P.band[k][b] % 128) return fail("band slot alignment", D, o, 0, 0);
         for (int k = 0; k < ops.KO; k++)
            if (P.own[k] % 16) return fail("own slot alignment", D, o, 0, 0);
         if (ops.KD && P.ownd[0] % 16) return fail("FP64 own slot alignment", D, o, 0, 0);
         if (!P.zero) return fail("offset 0 not found", D, o, 0, 0);
         for (const int64_t n : sizes) {
            const int64_t npad = (n + 3) / 4 * 4;   // vectors read by runs
            const int64_t pitch = (n + 7) / 8 * 8;  // rows of a value run
            const int64_t tiles = (n + kBandT - 1) / kBandT;
            for (int64_t t = 0; t < tiles; t++) {
               const int64_t i0 = t * kBandT;
               const int64_t vrows = pitch - i0 < kBandT ? pitch - i0 : kBandT;
               if ((vrows * ops.vbytes) % 16 || (pitch * ops.vbytes) % 16 || (i0 * ops.vbytes) % 16)
                  return fail("value run alignment", D, o, n, i0);
               const int64_t orows = npad - i0 < kBandT ? npad - i0 : kBandT;
               if ((orows * 4) % 16 || (i0 * 4) % 16) return fail("own run alignment", D, o, n, i0);
               // the value runs, then the own-row runs, fit before the
               // next part of the stage
               const uint32_t after_vals = ops.KB ? P.band[0][0] : ops.KO ? P.own[0] : ops.KD ? P.ownd[0] : P.bytes;
               if ((int64_t)P.vals + (int64_t)(D - 1) * kBandT * ops.vbytes + vrows * ops.vbytes > after_vals)
                  return fail("value runs exceed their slots", D, o, n, i0);
               for (int k = 0; k < ops.KO; k++) {
                  const uint32_t end = k + 1 < ops.KO ? P.own[k + 1] : ops.KD ? P.ownd[0] : P.bytes;
                  if ((int64_t)P.own[k] + 4 * orows > (int64_t)end) return fail("own run exceeds its slot", D, o, n, i0);
               }
               if (ops.KD && (int64_t)P.ownd[0] + 8 * orows > (int64_t)P.bytes)
                  return fail("FP64 own run exceeds its slot", D, o, n, i0);
               int64_t gs[8], ge[8];
               for (int b = 0; b < P.nb; b++) {
                  gs[b] = run_start(P.lo[b], i0);
                  const int64_t e = (i0 + kBandT + P.hi[b] + 3) & ~(int64_t)3;
                  ge[b] = e > npad ? npad : e;
                  if (ge[b] > gs[b]) {
                     if (gs[b] % 4 || ge[b] % 4) return fail("band run alignment", D, o, n, i0);
                     // the slot of input k's run of band b ends where the
                     // next part of the stage begins
                     for (int k = 0; k < ops.KB; k++) {
                        const uint32_t end = b + 1 < P.nb ? P.band[k][b + 1]
                                             : k + 1 < ops.KB ? P.band[k + 1][0]
                                             : ops.KO ? P.own[0]
                                             : ops.KD ? P.ownd[0]
                                                      : P.bytes;
                        if ((int64_t)P.band[k][b] + 4 * (ge[b] - gs[b]) > (int64_t)end)
                           return fail("band run exceeds its slot", D, o, n, i0);
                     }
                  }
               }
               const bool interior = i0 + P.minlo >= 0 && i0 + kBandT + P.maxhi <= n && i0 + kBandT <= n;
               for (int j = 0; j < D; j++) {
                  int b = 0;
                  while (b + 1 < P.nb && P.lo[b + 1] <= o[j]) b++;
                  if (o[j] < P.lo[b] || o[j] > P.hi[b] || P.dlo[j] != P.lo[b])
                     return fail("diagonal outside its band", D, o, n, i0);
                  // every in-range column of the tile's rows lies in the run
                  const int64_t rend = i0 + kBandT < n ? i0 + kBandT : n;
                  int64_t cmin = i0 + o[j], cmax = rend - 1 + o[j];
                  if (cmin < 0) cmin = 0;
                  if (cmax > n - 1) cmax = n - 1;
                  if (cmin <= cmax && (cmin < gs[b] || cmax >= ge[b]))
                     return fail("a column outside the band run", D, o, n, i0);
                  if (interior)
                     for (int k = 0; k < ops.KB; k++)
                        if ((int64_t)P.xoff[k][j] != (int64_t)P.band[k][b] + 4 * (i0 + o[j] - gs[b]))
                           return fail("interior offset", D, o, n, i0);
               }
               if (interior)
                  for (int k = 0; k < ops.KB; k++) {
                     int b = 0;
                     while (b + 1 < P.nb && P.lo[b + 1] <= 0) b++;
                     if ((int64_t)P.selfoff[k] != (int64_t)P.band[k][b] + 4 * (i0 - gs[b]))
                        return fail("interior own offset", D, o, n, i0);
                  }
               cases++;
            }
         }
      }
   }
   std::printf("ok %ld\n", cases);
   return 0;
}
