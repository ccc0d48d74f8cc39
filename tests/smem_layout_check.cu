// Host-only check of the staged kernel's shared-memory carve (WindowSmem):
// every field aligned for its widest access -- 16 bytes for the metadata
// broadcasts, the key rows, the source records and the persistent kernel's
// int4 current item -- over the table shapes the library accepts (ring rows
// up to 8,192 samples, 1-200 active stations, FP32 and 16-bit rows, one or
// WS key rows).  Exit status = number of violations (0: pass).
#include <cstdio>
#include "bp_kernels.cuh"

template <int P, int KS, int MT, int WS, int SPS, bool MAXRED>
int check() {
  int bad = 0;
  for (int rowcap = 64; rowcap <= 8192; rowcap += 64)
    for (int active = 1; active <= 200; ++active)
      for (int rf = 1; rf <= 2; ++rf)
        for (int rows : {1, WS}) {
          const bp::WindowSmem<P, KS, MT, WS, 4, SPS, MAXRED> L(rowcap, active, rf, rows);
          if (L.meta % 16 || L.red % 16 || L.srci % 16 || L.bars % 16 || L.misc % 16 ||
              L.total % 128) {
            if (++bad <= 3) printf("P=%d KS=%d MT=%d rowcap=%d active=%d\n", P, KS, MT, rowcap,
                                   active);
          }
        }
  return bad;
}

int main() {
  int bad = 0;
  bad += check<1, 8, 8, 8, 1, true>() + check<2, 4, 16, 16, 1, true>();
  bad += check<2, 4, 16, 16, 2, true>() + check<3, 8, 8, 8, 2, true>();
  bad += check<4, 2, 32, 16, 2, true>() + check<2, 8, 16, 8, 2, false>();
  bad += check<3, 2, 16, 16, 2, false>() + check<4, 8, 16, 8, 1, true>();
  printf("violations: %d\n", bad);
  return bad > 255 ? 255 : bad;
}
