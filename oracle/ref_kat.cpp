// ref_kat.cpp -- known-answer dump from the reference's own compiled RNG and
// erflib objects (oracle/_ref/libdpsnn_refkat.a, built by `make ref`).
// TEST INFRASTRUCTURE ONLY: run by tests/golden/make_golden.py to pin the
// restatement's ran3/NormDev/LUT against the reference.
// Output: one "name index value" line per number, values as %a.
#include <cstdio>
#include "randdev.h"
#include "erflib.h"

int main() {
  randdevClass r;
  const int seeds[] = {1, 2, 7, 1250, 0};   // 0 last: continues the stream
  for (int s : seeds) {
    r.SetRandomSeed(s);
    for (int i = 0; i < 200; i++) printf("ran3_%d %d %a\n", s, i, r.Random());
  }
  r.SetRandomSeed(3);
  for (int i = 0; i < 101; i++) printf("normdev_3 %d %a\n", i, r.NormDev());
  erflibClass e;
  double lut[256];
  e.makeGaussianLUT(lut, 256, (double)0.3f, (double)(0.3f * 0.1f), 0.0, 2.0 * 0.3f);
  for (int i = 0; i < 256; i++) printf("lut_0.3 %d %a\n", i, lut[i]);
  const double rr[] = {-0.5, 0.0, 0.49999999999999994, 0.5, 1.5, 2.5, 18.5, 19.4999};
  for (int i = 0; i < 8; i++) printf("roundr2i %d %a\n", i, (double)e.roundr2i(rr[i]));
  return 0;
}
