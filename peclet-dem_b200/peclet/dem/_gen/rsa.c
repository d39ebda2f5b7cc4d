/* Random sequential addition of spheres for the synthetic benchmark scenes.
 *
 * Spheres are proposed in the given order (callers pass them largest first) at uniform random
 * positions inside [lo, hi] (kept one radius from closed walls; wrapped on periodic axes) and
 * rejected while they overlap an already placed sphere; each sphere gets at most `tries`
 * proposals. A uniform grid with cell edge >= the largest diameter holds the placed spheres as
 * linked lists. The generator is splitmix64 seeded with `seed`, so a scene is reproducible
 * bit for bit on any machine. Returns the number of spheres placed; placed[i] = 0 for the others.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

static uint64_t sm64(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
static double unit(uint64_t* s) { return (double)(sm64(s) >> 11) * (1.0 / 9007199254740992.0); }

/* region 0: the whole box; region 1: the part of a cylinder (axis z, radius rg[0], centre x = rg[1],
 * y = rg[2]) with y <= rg[3], each sphere lying entirely inside it */
static int inRegion(int region, const double* rg, const double* p, double r) {
  if (region == 0)
    return 1;
  const double dx = p[0] - rg[1], dy = p[1] - rg[2];
  return sqrt(dx * dx + dy * dy) + r <= rg[0] && p[1] + r <= rg[3];
}

static long rsa(long n, const double* r, const double* lo, const double* hi, const int* periodic,
                unsigned long long seed, int tries, int region, const double* rg, double* pos,
                unsigned char* placed);

long pdem_rsa_spheres(long n, const double* r, const double* lo, const double* hi, const int* periodic,
                      unsigned long long seed, int tries, double* pos, unsigned char* placed) {
  return rsa(n, r, lo, hi, periodic, seed, tries, 0, NULL, pos, placed);
}
long pdem_rsa_spheres_region(long n, const double* r, const double* lo, const double* hi, unsigned long long seed,
                             int tries, int region, const double* rg, double* pos, unsigned char* placed) {
  const int closed[3] = {0, 0, 0};
  return rsa(n, r, lo, hi, closed, seed, tries, region, rg, pos, placed);
}

static long rsa(long n, const double* r, const double* lo, const double* hi, const int* periodic,
                unsigned long long seed, int tries, int region, const double* rg, double* pos,
                unsigned char* placed) {
  double rmax = 0.0, ext[3];
  for (long i = 0; i < n; ++i)
    if (r[i] > rmax)
      rmax = r[i];
  int dims[3];
  double cell[3];
  for (int a = 0; a < 3; ++a) {
    ext[a] = hi[a] - lo[a];
    dims[a] = (int)floor(ext[a] / (2.0 * rmax));
    if (dims[a] < 1)
      dims[a] = 1;
    cell[a] = ext[a] / dims[a];
  }
  const long ncell = (long)dims[0] * dims[1] * dims[2];
  long* head = (long*)malloc(sizeof(long) * ncell);
  long* next = (long*)malloc(sizeof(long) * (n > 0 ? n : 1));
  for (long c = 0; c < ncell; ++c)
    head[c] = -1;
  uint64_t st = seed;
  long count = 0;
  for (long i = 0; i < n; ++i) {
    placed[i] = 0;
    for (int t = 0; t < tries; ++t) {
      double p[3];
      int c[3];
      for (int a = 0; a < 3; ++a) {
        const double lo2 = periodic[a] ? lo[a] : lo[a] + r[i];
        const double hi2 = periodic[a] ? hi[a] : hi[a] - r[i];
        p[a] = lo2 + unit(&st) * (hi2 - lo2);
        c[a] = (int)((p[a] - lo[a]) / cell[a]);
        if (c[a] >= dims[a])
          c[a] = dims[a] - 1;
        if (c[a] < 0)
          c[a] = 0;
      }
      int ok = inRegion(region, rg, p, r[i]);
      for (int dz = -1; dz <= 1 && ok; ++dz)
        for (int dy = -1; dy <= 1 && ok; ++dy)
          for (int dx = -1; dx <= 1 && ok; ++dx) {
            int q[3] = {c[0] + dx, c[1] + dy, c[2] + dz};
            int skip = 0;
            for (int a = 0; a < 3; ++a) {
              if (q[a] < 0 || q[a] >= dims[a]) {
                if (!periodic[a] || dims[a] < 3) {
                  if (!periodic[a])
                    skip = 1;
                }
                q[a] = (q[a] % dims[a] + dims[a]) % dims[a];
              }
            }
            if (skip)
              continue;
            for (long j = head[((long)q[2] * dims[1] + q[1]) * dims[0] + q[0]]; j >= 0; j = next[j]) {
              double d2 = 0.0;
              for (int a = 0; a < 3; ++a) {
                double d = pos[3 * j + a] - p[a];
                if (periodic[a])
                  d -= ext[a] * nearbyint(d / ext[a]);
                d2 += d * d;
              }
              const double rr = r[i] + r[j];
              if (d2 < rr * rr) {
                ok = 0;
                break;
              }
            }
          }
      if (ok) {
        for (int a = 0; a < 3; ++a)
          pos[3 * i + a] = p[a];
        const long k = ((long)c[2] * dims[1] + c[1]) * dims[0] + c[0];
        next[i] = head[k];
        head[k] = i;
        placed[i] = 1;
        ++count;
        break;
      }
    }
  }
  free(head);
  free(next);
  return count;
}
