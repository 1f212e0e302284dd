/* logf_fixup.c -- builds the table that makes the engine's logf equal to the
 * host C library's logf on every float in (0,1].
 *
 * For each float x in (0,1] it compares the C library's logf(x) with the
 * correctly rounded float log that dd_math.cuh computes (logf_cr_from with
 * the C library's double log as the one-ulp approximation), and lists the
 * inputs where they differ, with the C library's value.
 * Output (binary, little endian): uint32 n, uint32 keys[n], float vals[n],
 * uint32 bucket[LOGF_FIX_NBUCKET].   Usage: logf_fixup <out.bin>          */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "dd_math.cuh"

int main(int argc, char **argv) {
  if (argc != 2) { fprintf(stderr, "usage: %s out.bin\n", argv[0]); return 2; }
  uint32_t cap = 1u << 20, n = 0;
  uint32_t *keys = malloc(cap * sizeof *keys);
  float *vals = malloc(cap * sizeof *vals);
  uint32_t *bucket = calloc(LOGF_FIX_NBUCKET, sizeof *bucket);
  for (uint32_t b = 0x30000000u; b <= 0x3F800000u; b++) {
    float x;
    memcpy(&x, &b, 4);
    float g = logf(x);
    float m = logf_cr_from(x, log((double)x));
    if (memcmp(&g, &m, 4) != 0) {
      if (n == cap) {
        cap *= 2;
        keys = realloc(keys, cap * sizeof *keys);
        vals = realloc(vals, cap * sizeof *vals);
      }
      keys[n] = b;
      vals[n] = g;
      n++;
    }
  }
  uint32_t i = 0;
  for (uint32_t bk = 0; bk < LOGF_FIX_NBUCKET; bk++) {
    while (i < n && (keys[i] >> 12) < bk + LOGF_FIX_BASE) i++;
    bucket[bk] = i;
  }
  FILE *f = fopen(argv[1], "wb");
  if (!f) { perror(argv[1]); return 1; }
  fwrite(&n, 4, 1, f);
  fwrite(keys, 4, n, f);
  fwrite(vals, 4, n, f);
  fwrite(bucket, 4, LOGF_FIX_NBUCKET, f);
  fclose(f);
  printf("%u fix-up entries\n", n);
  return 0;
}
